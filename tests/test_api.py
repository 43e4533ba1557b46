"""Drop-in API semantics on the CPU: signatures, connect rules, transformation folding."""

import numpy
import pytest

from reikna_b200 import _native as N
from reikna_b200 import transformations as tr
from reikna_b200.core import Annotation, ArrayMetadata, Parameter, Transformation, Type
from reikna_b200.fft import FFT, FFTShift


def meta(shape, dtype=numpy.complex64):
    return ArrayMetadata(shape, dtype)


def names(comp):
    return list(comp.signature.parameters)


def test_typecheck():
    # reikna tests/test_fft/test_fft.py:139
    with pytest.raises(ValueError, match="FFT computation requires array of a complex dtype"):
        FFT(ArrayMetadata(100, numpy.float32))


def test_default_signature():
    fft = FFT(meta((4, 8)))
    assert names(fft) == ["output", "input", "inverse"]
    assert fft.signature.parameters["inverse"].default == 0
    assert fft.parameter.output.shape == (4, 8)


def test_trivial_connect_signature():
    # reikna tests/test_fft/test_fft.py:173-190
    arr = meta((128, 1, 1, 128))
    fft = FFT(arr, axes=(1, 2))
    scale = tr.mul_param(arr, numpy.int32)
    fft.parameter.input.connect(scale, scale.output, input_prime=scale.input, param=scale.param)
    assert names(fft) == ["output", "input_prime", "param", "inverse"]
    d = fft.describe()
    assert [p["note"] for p in d["passes"]] == ["copy"]


def test_connect_returns_computation_and_is_chainable():
    arr = meta((16,))
    fft = FFT(arr)
    t1 = tr.mul_const(arr, 2.0)
    t2 = tr.div_param(arr, numpy.float32)
    res = fft.parameter.output.connect(t1, t1.input, out1=t1.output)
    assert res is fft
    fft.parameter.out1.connect(t2, t2.input, out2=t2.output, scale=t2.param)
    assert names(fft) == ["out2", "scale", "input", "inverse"]
    d, ispec, ospec, scalars, _ = fft.native_descriptor()
    assert scalars == ["scale"]
    assert d.output.scale_re == 2.0 and d.output.scale_div_slot == 0


def test_connect_errors():
    arr = meta((16,))
    fft = FFT(arr)
    t = tr.mul_const(arr, 2.0)
    with pytest.raises(ValueError, match="is not a part of the signature"):
        fft.connect("nope", t, t.output, x=t.input)
    fft.parameter.input.connect(t, t.output, new_input=t.input)
    t2 = tr.mul_const(arr, 3.0)
    with pytest.raises(ValueError, match="hidden by transformations"):
        fft.connect("new_input", t2, t2.output, input=t2.input)
    t3 = tr.mul_const(meta((8,)), 3.0)
    with pytest.raises(ValueError, match="Incompatible types"):
        fft.connect("new_input", t3, t3.output, nn=t3.input)
    t4 = tr.copy(arr)
    with pytest.raises(ValueError, match="is not an output node"):
        fft.connect("new_input", t4, t4.input, nn=t4.output)


def test_external_names_cannot_start_with_underscore():
    arr = meta((16,))
    fft = FFT(arr)
    t = tr.copy(arr)
    with pytest.raises(ValueError, match="underscore"):
        fft.parameter.input.connect(t, t.output, _x=t.input)


def test_real_to_complex_fold():
    # examples/demo_real_to_complex_fft.py:20-46
    x = ArrayMetadata((3000,), numpy.float32)
    trf = tr.real_to_complex(x)
    fft = FFT(trf.parameter.output)
    fft.parameter.input.connect(trf, trf.parameter.output, new_input=trf.parameter.input)
    assert names(fft) == ["output", "new_input", "inverse"]
    d, ispec, *_ = fft.native_descriptor()
    assert d.input.format == N.FMT_F32 and ispec.arrays == ["new_input"]


def test_fftshift_fold_sets_output_shift():
    arr = meta((6, 7))
    fft = FFT(arr)
    sh = tr.fftshift(arr)
    fft.parameter.output.connect(sh, sh.input, new_output=sh.output)
    d, *_ = fft.native_descriptor()
    assert list(d.output.shift)[:2] == [3, 3]
    ish = tr.fftshift(arr, inverse=True)
    fft2 = FFT(arr)
    fft2.parameter.output.connect(ish, ish.input, new_output=ish.output)
    d2, *_ = fft2.native_descriptor()
    assert list(d2.output.shift)[:2] == [3, 4]


def test_split_and_combine_fold():
    arr = meta((32,))
    fft = FFT(arr)
    cc = tr.combine_complex(arr)
    sc = tr.split_complex(arr)
    fft.parameter.input.connect(cc, cc.output, in_re=cc.real, in_im=cc.imag)
    fft.parameter.output.connect(sc, sc.input, out_re=sc.real, out_im=sc.imag)
    assert names(fft) == ["out_re", "out_im", "in_re", "in_im", "inverse"]
    d, ispec, ospec, *_ = fft.native_descriptor()
    assert d.input.format == N.FMT_F32_PAIR and d.output.format == N.FMT_F32_PAIR
    assert ispec.arrays == ["in_re", "in_im"] and ospec.arrays == ["out_re", "out_im"]


def test_spectrogram_chain_fold():
    # examples/demo_specgram.py:196-254
    sig = ArrayMetadata((4096,), numpy.float32)
    frame = tr.rolling_frame(sig, 1024, 768, None)
    fft_arr = ArrayMetadata(frame.parameter.output.shape, numpy.complex64)
    real_arr = ArrayMetadata(frame.parameter.output.shape, numpy.float32)
    win = tr.hanning_window(real_arr, 1024)
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
    fft.parameter.amplitude.connect(crop, crop.parameter.input, cropped_amplitude=crop.parameter.output)
    assert names(fft) == ["cropped_amplitude", "flat_input", "inverse"]
    d, ispec, ospec, *_ = fft.native_descriptor()
    assert d.input.format == N.FMT_F32
    assert list(d.input.strides)[:2] == [256, 1]
    assert list(d.input.shape)[:2] == [13, 1024]
    assert d.input.window == N.WIN_HANN and d.input.window_len == 1024
    assert d.output.format == N.FMT_F32 and d.output.post == N.POST_NORM and d.output.post_param == 1.0
    assert list(d.output.shape)[:2] == [13, 513]


def test_code_only_transformation_becomes_a_compiled_edge():
    arr = meta((16,))
    t = Transformation(
        [Parameter("output", Annotation(arr, "o")), Parameter("input", Annotation(arr, "i"))],
        "${output.store_same}(${input.load_same});",
    )
    fft = FFT(arr)
    fft.parameter.input.connect(t, t.output, x=t.input)
    d, ispec, *_ = fft.native_descriptor()
    assert d.input.format == N.FMT_USER and ispec.kind == "user" and ispec.arrays == []
    # a built-in the code chains cannot mix in is refused with a clear message
    fft2 = FFT(arr)
    t2 = Transformation(
        [Parameter("output", Annotation(arr, "o")), Parameter("input", Annotation(arr, "i"))],
        "${output.store_same}(${input.load_same});",
    )
    fft2.parameter.input.connect(t2, t2.output, x=t2.input)
    w = tr.hanning_window(arr, 16)
    fft2.parameter.x.connect(w, w.output, y=w.input)
    with pytest.raises(NotImplementedError, match="chain with transformation code"):
        fft2.native_descriptor()


def test_type_from_value_and_annotation_roles():
    t = Type.from_value(numpy.zeros((3, 4), numpy.complex64))
    assert t.shape == (3, 4) and t.strides == (32, 8)
    assert Annotation(t).role == "io"
    assert Annotation(numpy.float32).role == "s"
    with pytest.raises(ValueError):
        Annotation(numpy.float32, "o")
    p = Parameter("x", Annotation(numpy.int32), default=3)
    assert p.default == 3 and p.rename("y").name == "y"


def test_torch_tensor_metadata():
    import torch

    x = torch.zeros(4, 6, dtype=torch.complex64)
    m = ArrayMetadata.from_arraylike(x)
    assert m.shape == (4, 6) and m.dtype == numpy.complex64 and m.strides == (48, 8)
    mt = ArrayMetadata.from_arraylike(x.t())
    assert mt.strides == (8, 48)
    fft = FFT(x)
    assert fft.describe()["passes"]


def test_fftshift_signature():
    s = FFTShift(meta((10, 11)), axes=(0, 1))
    assert names(s) == ["output", "input", "inverse"]


# ---- the whole built-in set folds into the edges ----------------------------------


def test_affine_chain_folds_constants():
    arr = meta((32,))
    fft = FFT(arr)
    a = tr.add_const(arr, 1 + 2j)
    m = tr.mul_const(arr, 3.0)
    # output -> add (1+2i) -> mul 3 -> leaf: leaf = 3 y + 3 (1 + 2i)
    fft.parameter.output.connect(a, a.input, o1=a.output)
    fft.parameter.o1.connect(m, m.input, o2=m.output)
    d, ispec, ospec, names_, scal = fft.native_descriptor()
    assert (d.output.scale_re, d.output.scale_im) == (3.0, 0.0)
    assert (d.output.add_re, d.output.add_im) == (3.0, 6.0) and d.output.add_slot == -1
    assert scal({}) == []


def test_affine_chain_with_runtime_scalars_uses_extra_slots():
    arr = meta((32,))
    fft = FFT(arr)
    mp = tr.mul_param(arr, numpy.complex64)
    ap = tr.add_param(arr, numpy.float32)
    # input chain: fft_in = p * (x + q)
    fft.parameter.input.connect(mp, mp.output, x1=mp.input, p=mp.param)
    fft.parameter.x1.connect(ap, ap.output, x=ap.input, q=ap.param)
    d, ispec, ospec, names_, scal = fft.native_descriptor()
    assert sorted(names_) == ["p", "q"]
    assert d.input.scale_slot == names_.index("p") and d.input.add_slot == 2
    vals = scal({"p": 2j, "q": 0.5})
    assert vals[names_.index("p")] == 2j and vals[2] == 1j


def test_constant_sources_and_sinks():
    arr = meta((16, 8))
    fft = FFT(arr)
    bc = tr.broadcast_param(arr)
    fft.parameter.input.connect(bc, bc.output, value=bc.param)
    ig = tr.ignore(arr)
    fft.parameter.output.connect(ig, ig.input)
    assert names(fft) == ["value", "inverse"]
    d, ispec, ospec, names_, scal = fft.native_descriptor()
    assert d.input.format == N.FMT_CONST and d.input.add_slot == 1 and ispec.arrays == []
    assert d.output.format == N.FMT_IGNORE and ospec.arrays == []
    assert scal({"value": 2 + 1j}) == [2 + 1j, 2 + 1j]
    assert fft.describe()["passes"]


def test_norm_param_and_copy_broadcasted():
    arr = meta((8, 16))
    fft = FFT(arr)
    npm = tr.norm_param(arr)
    fft.parameter.output.connect(npm, npm.input, mag=npm.output, order=npm.order)
    row = ArrayMetadata((16,), numpy.complex64)
    cb = tr.copy_broadcasted(row, arr)
    fft.parameter.input.connect(cb, cb.output, row=cb.input)
    d, ispec, *_ = fft.native_descriptor()
    assert d.output.post == N.POST_NORM and d.output.post_slot == 0
    assert list(d.input.strides)[:2] == [0, 1] and list(d.input.shape)[:2] == [8, 16]
