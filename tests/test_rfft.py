"""Half-length RFFT / IRFFT (reikna examples/demo_specialized_fft.py) against numpy.

The example's own check is atol = rtol = 1e-4 against numpy's rfft / irfft
(demo_specialized_fft.py:627-662); the tests also hold the complex64 rel-L2 bound.
"""

import numpy
import pytest

from helpers import fft_bound, rel_l2


def test_rfft_signatures_and_errors():
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import IRFFT, RFFT

    r = RFFT(ArrayMetadata((8, 100), numpy.float32))
    assert tuple(r.parameter.output.shape) == (8, 51) and r.parameter.output.dtype == numpy.complex64
    r = RFFT(ArrayMetadata((100,), numpy.float64), dont_store_last=True)
    assert tuple(r.parameter.output.shape) == (50,) and r.parameter.output.dtype == numpy.complex128
    i = IRFFT(ArrayMetadata((8, 51), numpy.complex64))
    assert tuple(i.parameter.output.shape) == (8, 100) and i.parameter.output.dtype == numpy.float32
    with pytest.raises(ValueError):
        RFFT(ArrayMetadata((8, 101), numpy.float32))
    with pytest.raises(ValueError):
        RFFT(ArrayMetadata((8, 100), numpy.complex64))
    with pytest.raises(ValueError):
        IRFFT(ArrayMetadata((8, 100), numpy.float32))


@pytest.mark.gpu
@pytest.mark.parametrize(
    "shape,dtype",
    [((64, 4096), numpy.float32), ((1000, 1000), numpy.float32), ((3, 16384), numpy.float64), ((5, 3000), numpy.float32),
     ((2,), numpy.float32), ((7, 2, 256), numpy.float32)],
)
def test_rfft_and_irfft(shape, dtype):
    import torch

    from reikna_b200.fft import IRFFT, RFFT

    rng = numpy.random.default_rng(61)
    x = rng.uniform(-1, 1, shape).astype(dtype)
    t = torch.from_numpy(x).cuda()
    cdt = torch.complex64 if dtype == numpy.float32 else torch.complex128
    ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
    n = shape[-1]
    spec = torch.empty(shape[:-1] + (n // 2 + 1,), dtype=cdt, device="cuda")
    RFFT(t).compile()(None, spec, t)
    back = torch.empty_like(t)
    IRFFT(spec).compile()(None, back, spec)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64), axis=-1)
    got = spec.cpu().numpy()
    assert rel_l2(got, ref) < fft_bound(ctype, n)
    assert numpy.allclose(got, ref, atol=1e-4 * max(1.0, numpy.abs(ref).max()), rtol=1e-4)
    y = back.cpu().numpy()
    assert rel_l2(y, x.astype(numpy.float64)) < 2 * fft_bound(ctype, n)
    assert numpy.allclose(y, numpy.fft.irfft(ref, n=n, axis=-1), atol=1e-4, rtol=1e-4)


@pytest.mark.gpu
def test_rfft_without_last_bin_and_irfft_ignores_imaginary_edges():
    import torch

    from reikna_b200.fft import IRFFT, RFFT

    rng = numpy.random.default_rng(62)
    x = rng.standard_normal((16, 512)).astype(numpy.float32)
    t = torch.from_numpy(x).cuda()
    spec = torch.empty((16, 256), dtype=torch.complex64, device="cuda")
    RFFT(t, dont_store_last=True).compile()(None, spec, t)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64))[:, :256]
    assert rel_l2(spec.cpu().numpy(), ref) < fft_bound(numpy.complex64, 512)
    full = numpy.fft.rfft(x.astype(numpy.float64)).astype(numpy.complex64)
    full[:, 0] += 3j
    full[:, -1] -= 2j
    s = torch.from_numpy(full).cuda()
    out = torch.empty((16, 512), dtype=torch.float32, device="cuda")
    IRFFT(s).compile()(None, out, s)
    torch.cuda.synchronize()
    assert numpy.allclose(out.cpu().numpy(), numpy.fft.irfft(full.astype(numpy.complex128)), atol=1e-4, rtol=1e-4)


def test_real_post_flag_plans_one_pass():
    from reikna_b200 import _native as N

    d = N.desc(N.FMT_C64, (64, 512), (1,), N.FLAG_REAL_POST)
    d.output = N.edge(N.FMT_C64, (64, 513))
    plan = N.describe(d)
    assert len(plan["passes"]) == 1 and plan["passes"][0]["var"] == 3
    d = N.desc(N.FMT_C64, (64, 500), (1,), N.FLAG_REAL_POST)
    with pytest.raises(NotImplementedError):
        N.describe(d)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dtype", [((16384, 1024), numpy.float32), ((4, 16384), numpy.float32), ((3, 8192), numpy.float64)])
def test_fused_rfft_is_one_launch(shape, dtype):
    import torch

    from reikna_b200.fft import RFFT

    rng = numpy.random.default_rng(63)
    x = rng.uniform(-1, 1, shape).astype(dtype)
    t = torch.from_numpy(x).cuda()
    cdt = torch.complex64 if dtype == numpy.float32 else torch.complex128
    for last in (False, True):
        n = shape[-1]
        spec = torch.empty(shape[:-1] + (n // 2 + (0 if last else 1),), dtype=cdt, device="cuda")
        c = RFFT(t, dont_store_last=last).compile()
        assert c.launches == 1
        c(None, spec, t)
        torch.cuda.synchronize()
        ref = numpy.fft.rfft(x.astype(numpy.float64))[..., : spec.shape[-1]]
        ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
        assert rel_l2(spec.cpu().numpy(), ref) < fft_bound(ctype, n)


def test_oracle_real_transforms_match_numpy():
    """The oracle's restatement of the example's reference functions agrees with numpy,
    as the example's own tests require (demo_specialized_fft.py:627-705)."""
    from oracle import oracle

    rng = numpy.random.default_rng(64)
    for dt in (numpy.float32, numpy.float64):
        half = rng.standard_normal((3, 512)).astype(dt)
        full = numpy.concatenate([half, -half], axis=-1).astype(numpy.float64)
        ref = numpy.fft.rfft(full)[:, 1::2]
        assert numpy.allclose(oracle.aprfft(half), ref, atol=1e-4, rtol=1e-4)
        f = (rng.standard_normal((3, 256)) + 1j * rng.standard_normal((3, 256))).astype(numpy.complex128)
        spec = numpy.zeros((3, 513), numpy.complex128)
        spec[:, 1::2] = f
        assert numpy.allclose(oracle.iaprfft(f), numpy.fft.irfft(spec)[:, :512], atol=1e-4, rtol=1e-4)
        x = rng.standard_normal((2, 1000)).astype(dt)
        assert numpy.allclose(oracle.rfft_half(x), numpy.fft.rfft(x.astype(numpy.float64)), atol=1e-4, rtol=1e-4)
        back = oracle.irfft_half(numpy.fft.rfft(x.astype(numpy.float64)))
        assert numpy.allclose(back, x, atol=1e-4, rtol=1e-4)


def test_antiperiodic_signatures_and_errors():
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import APRFFT, IAPRFFT

    a = APRFFT(ArrayMetadata((8, 512), numpy.float32))
    assert tuple(a.parameter.output.shape) == (8, 256) and a.parameter.output.dtype == numpy.complex64
    i = IAPRFFT(ArrayMetadata((8, 256), numpy.complex128))
    assert tuple(i.parameter.output.shape) == (8, 512) and i.parameter.output.dtype == numpy.float64
    with pytest.raises(ValueError):
        APRFFT(ArrayMetadata((8, 511), numpy.float32))
    with pytest.raises(ValueError):
        APRFFT(ArrayMetadata((8, 512), numpy.complex64))
    with pytest.raises(ValueError):
        IAPRFFT(ArrayMetadata((8, 256), numpy.float32))


def test_real_pre_and_antiperiodic_flags_plan_one_pass():
    from reikna_b200 import _native as N

    cases = [(N.FLAG_REAL_PRE, 513, 512, 4), (N.FLAG_REAL_POST | N.FLAG_ANTIPERIODIC, 512, 512, 3),
             (N.FLAG_REAL_PRE | N.FLAG_ANTIPERIODIC, 512, 512, 4)]
    for flags, n_in, n_out, var in cases:
        d = N.desc(N.FMT_C64, (64, 512), (1,), flags)
        d.input = N.edge(N.FMT_C64, (64, n_in))
        d.output = N.edge(N.FMT_C64, (64, n_out))
        plan = N.describe(d)
        assert len(plan["passes"]) == 1 and plan["passes"][0]["var"] == var
    # the inverse reads L + 1 bins, the antiperiodic transforms L harmonics
    for flags, n_in, n_out in [(N.FLAG_REAL_PRE, 512, 512), (N.FLAG_REAL_POST | N.FLAG_ANTIPERIODIC, 512, 513),
                               (N.FLAG_REAL_PRE | N.FLAG_ANTIPERIODIC, 513, 512)]:
        d = N.desc(N.FMT_C64, (64, 512), (1,), flags)
        d.input = N.edge(N.FMT_C64, (64, n_in))
        d.output = N.edge(N.FMT_C64, (64, n_out))
        with pytest.raises(NotImplementedError):
            N.describe(d)
    for flags in (N.FLAG_ANTIPERIODIC, N.FLAG_REAL_POST | N.FLAG_REAL_PRE):
        with pytest.raises(ValueError):
            N.describe(N.desc(N.FMT_C64, (64, 512), (1,), flags))


@pytest.mark.gpu
@pytest.mark.parametrize(
    "shape,dtype",
    [((512,), numpy.float32), ((64, 1024), numpy.float32), ((3, 8192), numpy.float64), ((2, 16), numpy.float32),
     ((2, 3, 512), numpy.float32), ((5, 1000), numpy.float32), ((2, 65536), numpy.float32), ((3, 600), numpy.float64)],
)
def test_aprfft_and_iaprfft(shape, dtype):
    """Against the oracle's restatement of the reference (atol = rtol = 1e-4, the example's
    own tolerance) and numpy in FP64 (the rel-L2 bound); the last three shapes have half
    lengths without a one-pass plan (Bluestein, four-step) and take the multi-kernel route."""
    import torch

    from oracle import oracle
    from reikna_b200.fft import APRFFT, IAPRFFT

    rng = numpy.random.default_rng(65)
    x = rng.standard_normal(shape).astype(dtype)
    ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
    cdt = torch.complex64 if dtype == numpy.float32 else torch.complex128
    n = shape[-1]
    t = torch.from_numpy(x).cuda()
    harm = torch.empty(shape[:-1] + (n // 2,), dtype=cdt, device="cuda")
    fwd = APRFFT(t).compile()
    fused = (n // 2) in [2**k for k in range(3, 14 if dtype == numpy.float32 else 13)]
    assert (fwd.launches == 1) == fused
    fwd(None, harm, t)
    back = torch.empty_like(t)
    inv = IAPRFFT(harm).compile()
    assert (inv.launches == 1) == fused
    inv(None, back, harm)
    torch.cuda.synchronize()
    got = harm.cpu().numpy()
    full = numpy.concatenate([x, -x], axis=-1).astype(numpy.float64)
    ref = numpy.fft.rfft(full, axis=-1)[..., 1::2]
    assert rel_l2(got, ref) < fft_bound(ctype, 2 * n)
    orc = oracle.aprfft(x)
    assert numpy.allclose(got, orc, atol=1e-4 * max(1.0, numpy.abs(orc).max()), rtol=1e-4)
    y = back.cpu().numpy()
    assert rel_l2(y, x.astype(numpy.float64)) < 2 * fft_bound(ctype, 2 * n)
    assert numpy.allclose(y, oracle.iaprfft(got.astype(numpy.complex128)), atol=1e-4, rtol=1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dtype", [((16384, 1024), numpy.float32), ((4, 16384), numpy.float32), ((3, 8192), numpy.float64)])
def test_fused_irfft_is_one_launch(shape, dtype):
    import torch

    from reikna_b200.fft import IRFFT

    rng = numpy.random.default_rng(66)
    n = shape[-1]
    ctype = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
    spec = numpy.fft.rfft(rng.uniform(-1, 1, shape)).astype(ctype)
    spec[..., 0] += 0.5j  # ignored, as numpy's irfft ignores it
    s = torch.from_numpy(spec).cuda()
    out = torch.empty(shape, dtype=torch.float32 if dtype == numpy.float32 else torch.float64, device="cuda")
    c = IRFFT(s).compile()
    assert c.launches == 1
    c(None, out, s)
    torch.cuda.synchronize()
    ref = numpy.fft.irfft(spec.astype(numpy.complex128), n=n, axis=-1)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(ctype, n)


@pytest.mark.gpu
def test_real_plans_run_in_their_direction_only():
    import torch

    from reikna_b200 import _native as N

    for flags, n_in, wrong in [(N.FLAG_REAL_POST, 256, 1), (N.FLAG_REAL_PRE, 257, 0),
                               (N.FLAG_REAL_POST | N.FLAG_ANTIPERIODIC, 256, 1), (N.FLAG_REAL_PRE | N.FLAG_ANTIPERIODIC, 256, 0)]:
        d = N.desc(N.FMT_C64, (4, 256), (1,), flags)
        d.input = N.edge(N.FMT_C64, (4, n_in))
        d.output = N.edge(N.FMT_C64, (4, 256))
        plan = N.Plan(d)
        a = torch.zeros((4, n_in), dtype=torch.complex64, device="cuda")
        b = torch.zeros((4, 256), dtype=torch.complex64, device="cuda")
        with pytest.raises(ValueError):
            plan.execute([b.data_ptr()], [a.data_ptr()], inverse=wrong, stream=0)
        plan.execute([b.data_ptr()], [a.data_ptr()], inverse=1 - wrong, stream=0)
    torch.cuda.synchronize()


def _r2c_crop_fft(meta_real, cdt, flags_note=None):
    from reikna_b200 import transformations as tr
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import FFT

    fft = FFT(ArrayMetadata(tuple(meta_real.shape), cdt), axes=(len(meta_real.shape) - 1,))
    scale = tr.mul_param(fft.parameter.input, cdt)
    fft.parameter.input.connect(scale, scale.parameter.output, scaled=scale.parameter.input, k=scale.parameter.param)
    r2c = tr.real_to_complex(meta_real)
    fft.parameter.scaled.connect(r2c, r2c.parameter.output, real=r2c.parameter.input)
    crop = tr.crop_frequencies(fft.parameter.output)
    fft.parameter.output.connect(crop, crop.parameter.input, half=crop.parameter.output)
    return fft


def test_real_input_with_cropped_output_plans_the_half_route():
    from reikna_b200.core import ArrayMetadata

    fft = _r2c_crop_fft(ArrayMetadata((37, 1024), numpy.float32), numpy.complex64)
    p = fft.describe()["passes"]
    assert len(p) == 1 and p[0]["note"] == "half" and p[0]["L"] == 512 and p[0]["var"] == 6
    # an odd length, or an output keeping the negative frequencies, keeps the full transform
    assert _r2c_crop_fft(ArrayMetadata((37, 1000), numpy.float32), numpy.complex64).describe()["passes"][0]["note"] != "half"
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    full = FFT(ArrayMetadata((37, 1024), numpy.complex64), axes=(1,))
    r2c = tr.real_to_complex(ArrayMetadata((37, 1024), numpy.float32))
    full.parameter.input.connect(r2c, r2c.parameter.output, real=r2c.parameter.input)
    assert full.describe()["passes"][0]["note"] != "half"


@pytest.mark.gpu
@pytest.mark.parametrize("rows,n,dtype", [(37, 1024, numpy.float32), (5, 8192, numpy.float64), (64, 16, numpy.float32),
                                          (3, 16384, numpy.float32)])
@pytest.mark.parametrize("inverse", [0, 1])
@pytest.mark.parametrize("offset", [0, 1])
def test_half_route_for_real_input(rows, n, dtype, inverse, offset):
    """A real input transformed along the last axis and cropped to n/2 + 1 bins runs as
    the half-length transform of its sample pairs; a complex runtime scale of the input
    and the inverse direction act through the store (the input is real).  offset 1
    starts every row on an odd sample (no paired vector loads)."""
    import torch

    from reikna_b200.core import ArrayMetadata

    cdt = numpy.complex64 if dtype == numpy.float32 else numpy.complex128
    rng = numpy.random.default_rng(67)
    x = rng.standard_normal((rows, n + offset)).astype(dtype)
    t = torch.from_numpy(x).cuda()[:, offset:]
    fft = _r2c_crop_fft(ArrayMetadata.from_arraylike(t), cdt)
    assert fft.describe()["passes"][0]["note"] == "half"
    out = torch.empty((rows, n // 2 + 1), dtype=torch.complex64 if cdt == numpy.complex64 else torch.complex128,
                      device="cuda")
    k = 0.75 - 1.5j
    fft.compile()(None, out, t, k=k, inverse=inverse)
    torch.cuda.synchronize()
    xs = x[:, offset:].astype(numpy.float64) * k
    ref = (numpy.fft.ifft if inverse else numpy.fft.fft)(xs, axis=1)[:, : n // 2 + 1]
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(cdt, n)
    # the same computation through the full-length route
    full = torch.empty_like(out)
    fft.compile(flags=2**9)(None, full, t, k=k, inverse=inverse)
    torch.cuda.synchronize()
    assert fft.compile(flags=2**9)._runner.plan.describe()["passes"][0]["note"] != "half"
    assert rel_l2(full.cpu().numpy(), ref) < fft_bound(cdt, n)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,keep", [((2, 3, 512), 257), ((40, 1024), 100), ((7, 64), 5)])
def test_half_route_batched_and_cropped(shape, keep):
    """Half-length route through the C-ABI: a real input with any batch dims, and an
    output keeping fewer than n/2 + 1 bins (its store takes the strided-map path)."""
    import torch

    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(68)
    x = rng.standard_normal(shape).astype(numpy.float32)
    n = shape[-1]
    d = N.desc(N.FMT_C64, shape, (len(shape) - 1,))
    d.input = N.edge(N.FMT_F32, shape)
    d.output = N.edge(N.FMT_C64, shape[:-1] + (keep,))
    plan = N.Plan(d)
    assert plan.describe()["passes"][0]["note"] == "half"
    t = torch.from_numpy(x).cuda()
    out = torch.zeros(shape[:-1] + (keep,), dtype=torch.complex64, device="cuda")
    plan.execute([out.data_ptr()], [t.data_ptr()], inverse=0, stream=0)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64), axis=-1)[..., :keep]
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
def test_half_route_transposed_complex_output():
    """Real frames to a bins-by-frames complex picture: the half-length pass with the
    lane-fastest store (variant 5) writing complex values."""
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(69)
    frames, n = 300, 256
    x = rng.standard_normal((frames, n)).astype(numpy.float32)
    fft = FFT(ArrayMetadata((frames, n), numpy.complex64), axes=(1,))
    r2c = tr.real_to_complex(ArrayMetadata((frames, n), numpy.float32))
    fft.parameter.input.connect(r2c, r2c.parameter.output, real=r2c.parameter.input)
    crop = tr.crop_frequencies(fft.parameter.output)
    fft.parameter.output.connect(crop, crop.parameter.input, half=crop.parameter.output)
    tp = tr.transpose_2d(crop.parameter.output)
    fft.parameter.half.connect(tp, tp.parameter.input, picture=tp.parameter.output)
    p = fft.describe()["passes"]
    assert len(p) == 1 and p[0]["note"] == "half" and p[0]["var"] == 5
    out = torch.empty((n // 2 + 1, frames), dtype=torch.complex64, device="cuda")
    fft.compile()(None, out, torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(x.astype(numpy.float64), axis=1).T
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
@pytest.mark.parametrize("antiperiodic", [False, True])
def test_real_post_plan_with_output_scale(antiperiodic):
    """A complex scale on the output edge of a one-pass real transform multiplies every
    stored bin, the separately stored Nyquist bin included."""
    import torch

    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(70)
    rows, n = 9, 512
    x = rng.standard_normal((rows, n)).astype(numpy.float32)
    half = n // 2
    flags = N.FLAG_REAL_POST | (N.FLAG_ANTIPERIODIC if antiperiodic else 0)
    bins = half if antiperiodic else half + 1
    d = N.desc(N.FMT_C64, (rows, half), (1,), flags)
    d.input = N.edge(N.FMT_C64, (rows, half))
    d.output = N.edge(N.FMT_C64, (rows, bins))
    d.output.scale_re, d.output.scale_im = 0.5, -0.25
    plan = N.Plan(d)
    t = torch.from_numpy(x).cuda()
    out = torch.zeros((rows, bins), dtype=torch.complex64, device="cuda")
    plan.execute([out.data_ptr()], [t.data_ptr()], inverse=0, stream=0)
    torch.cuda.synchronize()
    if antiperiodic:
        ref = numpy.fft.rfft(numpy.concatenate([x, -x], axis=1).astype(numpy.float64), axis=1)[:, 1::2]
    else:
        ref = numpy.fft.rfft(x.astype(numpy.float64), axis=1)
    ref = ref * (0.5 - 0.25j)
    assert rel_l2(out.cpu().numpy(), ref) < fft_bound(numpy.complex64, 2 * n)
    if not antiperiodic:
        assert numpy.allclose(out.cpu().numpy()[:, -1], ref[:, -1], atol=1e-3 * numpy.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("antiperiodic", [False, True])
def test_real_pre_plan_with_input_scale(antiperiodic):
    """A complex scale on the input edge of a one-pass inverse real transform acts on the
    spectrum before the real step (numpy's irfft of the scaled spectrum: the imaginary
    parts of bins 0 and L are dropped after scaling)."""
    import torch

    from reikna_b200 import _native as N

    rng = numpy.random.default_rng(71)
    rows, half = 6, 256
    c = 0.5 - 0.25j
    if antiperiodic:
        f = (rng.standard_normal((rows, half)) + 1j * rng.standard_normal((rows, half))).astype(numpy.complex64)
        spec = numpy.zeros((rows, 2 * half + 1), numpy.complex128)
        spec[:, 1::2] = f * c
        ref = numpy.fft.irfft(spec, axis=1)[:, : 2 * half]
        bins = half
    else:
        f = (rng.standard_normal((rows, half + 1)) + 1j * rng.standard_normal((rows, half + 1))).astype(numpy.complex64)
        ref = numpy.fft.irfft(f.astype(numpy.complex128) * c, axis=1)
        bins = half + 1
    flags = N.FLAG_REAL_PRE | (N.FLAG_ANTIPERIODIC if antiperiodic else 0)
    d = N.desc(N.FMT_C64, (rows, half), (1,), flags)
    d.input = N.edge(N.FMT_C64, (rows, bins))
    d.output = N.edge(N.FMT_C64, (rows, half))
    d.input.scale_re, d.input.scale_im = c.real, c.imag
    plan = N.Plan(d)
    s = torch.from_numpy(f).cuda()
    out = torch.zeros((rows, 2 * half), dtype=torch.float32, device="cuda")
    plan.execute([out.data_ptr()], [s.data_ptr()], inverse=1, stream=0)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) < 2 * fft_bound(numpy.complex64, 2 * half)


@pytest.mark.gpu
@pytest.mark.parametrize("offset", [0, 1])
def test_rfft_of_any_view(offset):
    """RFFT reads the real array through the half-length route's sample-pair loads, so a
    contiguous view starting on an odd sample works (scalar loads for its lines)."""
    import torch

    from reikna_b200.fft import RFFT

    rng = numpy.random.default_rng(72)
    flat = rng.standard_normal(33 * 1024 + offset).astype(numpy.float32)
    t = torch.from_numpy(flat).cuda()[offset:].view(33, 1024)  # contiguous, odd start for offset 1
    spec = torch.empty((33, 513), dtype=torch.complex64, device="cuda")
    c = RFFT(t).compile()
    assert c.launches == 1
    c(None, spec, t)
    torch.cuda.synchronize()
    ref = numpy.fft.rfft(flat[offset:].reshape(33, 1024).astype(numpy.float64), axis=1)
    assert rel_l2(spec.cpu().numpy(), ref) < fft_bound(numpy.complex64, 1024)
