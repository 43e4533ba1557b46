"""Batched execution (one persistent launch, CUDA-graph replay with and without one
branch per member, plain calls).

Batched results must be bit-identical to the same members run one call at a time with
the same plan flags: the tile bodies are the same device code with the same
parameters.  Against numpy they meet the usual bound.
"""

import json

import numpy
import pytest

from helpers import fft_bound, normal_array, rel_l2


def _c3_members(torch):
    """The three mixed-size members of the batched configuration: 1000x3001 Bluestein
    (axis 1), 1000x1000 over both axes, and a 1000x1000 real-to-complex transform
    cropped to 1000x501."""
    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    rng4, rng5, rng6 = (numpy.random.default_rng(s) for s in (4, 5, 6))
    xa = normal_array(rng4, (1000, 3001), numpy.complex64)
    xb = normal_array(rng5, (1000, 1000), numpy.complex64)
    xc = rng6.uniform(-1, 1, (1000, 1000)).astype(numpy.float32)
    ta, tb, tc = (torch.from_numpy(x).cuda() for x in (xa, xb, xc))
    fa = FFT(ta, axes=(1,))
    fb = FFT(tb, axes=(0, 1))
    r2c = tr.real_to_complex(tc)
    fc = FFT(r2c.parameter.output)
    fc.parameter.input.connect(r2c, r2c.parameter.output, real_input=r2c.parameter.input)
    crop = tr.crop_frequencies(fc.parameter.output)
    fc.parameter.output.connect(crop, crop.parameter.input, half=crop.parameter.output)
    outs = [torch.empty_like(ta), torch.empty_like(tb), torch.empty((1000, 501), dtype=torch.complex64, device="cuda")]
    refs = [
        numpy.fft.fft(xa.astype(numpy.complex128), axis=1),
        numpy.fft.fft2(xb.astype(numpy.complex128)),
        numpy.fft.rfft2(xc.astype(numpy.float64)),
    ]
    sizes = [3001, 10**6, 10**6]
    return [fa, fb, fc], [ta, tb, tc], outs, refs, sizes


# --- host-side logic (no GPU) ----------------------------------------------------


def test_unknown_mode_rejected():
    from reikna_b200.batch import BatchedFFT

    with pytest.raises(ValueError, match="unknown batch mode"):
        BatchedFFT([object()], mode="fastest")


def test_autotune_cache_roundtrip(tmp_path, monkeypatch):
    from reikna_b200 import batch

    monkeypatch.setenv("RK_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    assert batch._load_cache() == {}
    batch._store_cache("k1", {"mode": "graph", "flags": 16, "ms": 0.5})
    batch._store_cache("k2", {"mode": "persistent", "flags": 1, "ms": 0.2})
    data = json.loads((tmp_path / "tune.json").read_text())
    assert data["k1"]["mode"] == "graph" and data["k2"]["flags"] == 1
    (tmp_path / "tune.json").write_text("{not json")
    assert batch._load_cache() == {}


def test_batch_key_depends_on_members():
    from reikna_b200 import _native as N
    from reikna_b200.batch import _desc_key

    a = N.desc(N.FMT_C64, (1000, 3001), (1,))
    b = N.desc(N.FMT_C64, (1000, 1000), (0, 1))
    assert _desc_key([a, b]) == _desc_key([a, b])
    assert _desc_key([a, b]) != _desc_key([b, a])


def test_branch_parallel_graph_is_a_candidate_for_several_members():
    import torch

    from reikna_b200.batch import MODES, BatchedFFT
    from reikna_b200.core import ArrayMetadata
    from reikna_b200.fft import FFT

    assert "graph_par" in MODES
    dev = torch.device("cuda", 0)  # no plan is compiled in mode "auto" before the first call
    a = FFT(ArrayMetadata((64, 1024), numpy.complex64), axes=(1,))
    b = FFT(ArrayMetadata((32, 32), numpy.complex64))
    modes = [m for m, _ in BatchedFFT([a, b], device=dev).candidates()]
    assert "graph_par" in modes and "graph" in modes and "persistent" in modes
    assert "graph_par" not in [m for m, _ in BatchedFFT([a], device=dev).candidates()]


# --- GPU ---------------------------------------------------------------------------


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["persistent", "graph", "graph_par", "calls"])
def test_batch_matches_single_calls(mode):
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.batch import BatchedFFT

    comps, ins, outs, refs, sizes = _c3_members(torch)
    bat = BatchedFFT(comps, mode=mode)
    flags = bat.chosen[1]
    for _ in range(2):  # second call reuses staging / graph
        for o in outs:
            o.zero_()
        bat(None, [(o, i) for o, i in zip(outs, ins)])
    torch.cuda.synchronize()
    got = [o.clone() for o in outs]
    singles = [c.compile(flags=flags) for c in comps]
    for s, o, i in zip(singles, outs, ins):
        o.zero_()
        s(None, o, i)
    torch.cuda.synchronize()
    for g, o, r, n in zip(got, outs, refs, sizes):
        assert torch.equal(g, o)
        assert rel_l2(g.cpu().numpy(), r) < fft_bound(numpy.complex64, n)
    assert N.device_status(clear=True) == 0
    bat.close()


@pytest.mark.gpu
def test_persistent_batch_info_and_pointer_change():
    import torch

    from reikna_b200.batch import BatchedFFT

    comps, ins, outs, refs, sizes = _c3_members(torch)
    bat = BatchedFFT(comps, mode="persistent")
    info = bat._variant.batch.info()
    assert info["passes"] == 1 + 5 + 5 and info["grid"] >= 148
    bat(None, [(o, i) for o, i in zip(outs, ins)])
    # new buffers: the per-call pointer upload must follow them
    outs2 = [torch.empty_like(o) for o in outs]
    ins2 = [i.clone() for i in ins]
    bat(None, [(o, i) for o, i in zip(outs2, ins2)])
    torch.cuda.synchronize()
    for a, b in zip(outs, outs2):
        assert torch.equal(a, b)


@pytest.mark.gpu
def test_persistent_batch_inverse_and_scalars():
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.batch import BatchedFFT
    from reikna_b200.fft import FFT

    rng = numpy.random.default_rng(21)
    shapes = [((64, 4096), (1,)), ((256, 512), (0,)), ((100, 200), (0, 1)), ((8, 1000), (1,))]
    comps, args, refs = [], [], []
    for k, (shape, axes) in enumerate(shapes):
        x = normal_array(rng, shape, numpy.complex64)
        t = torch.from_numpy(x).cuda()
        f = FFT(t, axes=axes)
        inverse = k % 2
        ref = (numpy.fft.ifftn if inverse else numpy.fft.fftn)(x.astype(numpy.complex128), axes=axes)
        if k == 2:
            m = tr.mul_param(f.parameter.output, numpy.complex64)
            f.parameter.output.connect(m, m.parameter.input, out=m.parameter.output, coeff=m.parameter.param)
            args.append({"out": torch.empty_like(t), "input": t, "coeff": 0.5 - 2j, "inverse": inverse})
            ref = ref * (0.5 - 2j)
        else:
            args.append({"output": torch.empty_like(t), "input": t, "inverse": inverse})
        comps.append(f)
        refs.append(ref)
    bat = BatchedFFT(comps, mode="persistent")
    bat(None, args)
    torch.cuda.synchronize()
    for (shape, axes), a, r in zip(shapes, args, refs):
        n = int(numpy.prod([shape[ax] for ax in axes]))
        res = a["out"] if "out" in a else a["output"]
        assert rel_l2(res.cpu().numpy(), r) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
def test_persistent_batch_rejects_unsupported_members():
    import torch

    from reikna_b200.batch import BatchedFFT
    from reikna_b200.fft import FFT

    t = torch.zeros((64, 64), dtype=torch.complex128, device="cuda")
    with pytest.raises(NotImplementedError, match="no batched variant"):
        BatchedFFT([FFT(t)], mode="persistent")


@pytest.mark.gpu
def test_native_batch_rejects_repeated_plan():
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    t = torch.zeros((64, 256), dtype=torch.complex64, device="cuda")
    c = FFT(t, axes=(1,)).compile()
    with pytest.raises(ValueError, match="appears twice"):
        N.Batch([c._runner.plan, c._runner.plan])


@pytest.mark.gpu
def test_autotuned_batch(tmp_path, monkeypatch):
    import torch

    from reikna_b200.batch import BatchedFFT

    monkeypatch.setenv("RK_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    comps, ins, outs, refs, sizes = _c3_members(torch)
    bat = BatchedFFT(comps)
    bat(None, [(o, i) for o, i in zip(outs, ins)])
    torch.cuda.synchronize()
    assert bat.tuning["cached"] is False and len(bat.tuning["tried"]) >= 4
    for o, r, n in zip(outs, refs, sizes):
        assert rel_l2(o.cpu().numpy(), r) < fft_bound(numpy.complex64, n)
    again = BatchedFFT(comps)
    again(None, [(o, i) for o, i in zip(outs, ins)])
    assert again.tuning["cached"] is True and again.chosen == bat.chosen
