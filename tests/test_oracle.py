"""The CPU oracle against reikna's own planner (golden fixtures) and numpy (CPU only)."""

import json
import math
from pathlib import Path

import numpy
import pytest

from helpers import FFT_ATOL, FFT_RTOL, diff_is_negligible, fft_bound, rel_l2, uniform_array
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
PLANNER = json.loads((GOLDEN / "planner.json").read_text())


@pytest.mark.parametrize("size", [2**k for k in range(1, 21)])
def test_radix_array_matches_reikna(size):
    g = PLANNER["radix"][str(size)]
    assert O.radix_array(size) == g["radix_array"]
    assert O.radix_array(size, use_max_radix=True) == g["radix_array_max"]


@pytest.mark.parametrize("size", [2**k for k in range(1, 25)])
def test_global_radix_info_matches_reikna(size):
    assert [list(x) for x in O.global_radix_info(size)] == PLANNER["radix"][str(size)]["global"]


def test_radix_array_rejects_non_pow2():
    with pytest.raises(ValueError):
        O.radix_array(12)


@pytest.mark.parametrize("name", sorted(numpy.load(GOLDEN / "kweights.npz").files))
def test_kweights_match_reikna(name):
    ref = numpy.load(GOLDEN / "kweights.npz")[name]
    n, m = (int(v) for v in name.split("_")[1:])
    kw = O.kweights(n, m)
    assert kw.shape == ref.shape
    scale = numpy.abs(ref).max()
    assert numpy.abs(kw - ref).max() / scale < 1e-9


@pytest.mark.parametrize("case", PLANNER["chains"], ids=lambda c: f"{c['shape']}-{c['axes']}")
def test_kernel_chain_matches_reikna(case):
    chain = O.kernel_chain(case["shape"], case["axes"], case["local_kernel_limit"])
    gold = case["kernels"]
    assert len(chain) == len(gold)
    for mine, ref in zip(chain, gold):
        assert mine["kind"] == ref["kind"]
        assert mine["fft_size"] == ref["fft_size"]
        assert mine["fft_size_real"] == ref["fft_size_real"]
        assert mine["radix"] == ref["radix"]
        assert mine["pass_num"] == ref["pass_num"]
        for f in ("reverse_direction", "pad_in", "unpad_out", "takes_kweights"):
            assert mine[f] == ref[f], f
        if ref["kind"] == "global":
            assert (mine["radix1"], mine["radix2"]) == (ref["radix1"], ref["radix2"])


# shape lists of reikna's own FFT tests (tests/test_fft/test_fft.py:44-111), with
# batches reduced so the CPU suite stays fast
LOCAL = [((b, s), (1,)) for p in (3, 7, 8, 9, 10, 12) for s in (2**p, 2**p // 2 - 1) for b in (1, 3)]
GLOBAL = [((ob, s, ib), (1,)) for p in (3, 7, 9) for s in (2**p, 2**p // 2 - 1) for ib in (2, 3, 63) for ob in (1, 2)]
SEQUENCE = [((3, 255, 7), (2, 0)), ((17, 200, 31), (1, 0)), ((7, 100, 11), (1, 2)), ((5, 90, 17), (2, 0, 1))]


@pytest.mark.parametrize("shape_axes", LOCAL + GLOBAL, ids=str)
@pytest.mark.parametrize("dtype", [numpy.complex64, numpy.complex128])
def test_oracle_against_numpy(rng, shape_axes, dtype):
    shape, axes = shape_axes
    x = uniform_array(rng, shape, dtype)
    n = math.prod(shape[a] for a in axes)
    for inverse in (False, True):
        y = O.fft(x, axes, inverse=inverse, threads=2)
        ref = O.numpy_ref(x, axes, inverse)
        assert rel_l2(y, ref) < fft_bound(dtype, n)
        if dtype == numpy.complex64:
            assert diff_is_negligible(y, ref.astype(dtype), FFT_ATOL, FFT_RTOL)


@pytest.mark.parametrize("shape_axes", SEQUENCE, ids=str)
def test_oracle_sequence(rng, shape_axes):
    shape, axes = shape_axes
    x = uniform_array(rng, shape, numpy.complex64)
    y = O.fft(x, axes, threads=2)
    ref = O.numpy_ref(x, axes)
    assert diff_is_negligible(y, ref.astype(numpy.complex64), FFT_ATOL, 1e-2)
    assert rel_l2(y, ref) < fft_bound(numpy.complex64, math.prod(shape[a] for a in axes))


def test_oracle_trivial_is_copy(rng):
    x = uniform_array(rng, (8, 1, 1, 8), numpy.complex64)
    assert numpy.array_equal(O.fft(x, (1, 2)), x)
