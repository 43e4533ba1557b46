"""Serving loop: grouping logic on the host, and on the GPU the same result for a
request whether it is served alone or in a mix of others (stated FP32 bound)."""

import numpy
import pytest

from helpers import fft_bound, rel_l2


def test_binary_pieces():
    from reikna_b200.serve import binary_pieces

    assert binary_pieces(1) == [1]
    assert binary_pieces(37) == [32, 4, 1]
    assert binary_pieces(256) == [256]
    for n in range(1, 600):
        p = binary_pieces(n)
        assert sum(p) == n and len(set(p)) == len(p) and all(x & (x - 1) == 0 for x in p)
    with pytest.raises(ValueError):
        binary_pieces(0)


def test_request_classes_and_bytes():
    import torch

    from reikna_b200.serve import FFTRequest, FFTServer

    a = FFTRequest("fft1d", torch.zeros((3, 1000), dtype=torch.complex64))
    b = FFTRequest("fft1d", torch.zeros((7, 1000), dtype=torch.complex64), inverse=1)
    c = FFTRequest("fft2d", torch.zeros((64, 48), dtype=torch.complex64))
    d = FFTRequest("spectrogram", torch.zeros(8192, dtype=torch.float32), nfft=256, hop=64)
    assert a.key() == ("fft1d", 1000, 0) and b.key() == ("fft1d", 1000, 1)
    assert c.key() == ("fft2d", 64, 48, 0) and d.key() == ("spectrogram", 8192, 256, 64)
    assert a.rows() == 3 and c.rows() == 1
    assert d.out_shape() == ((8192 - 192) // 64, 129)
    assert FFTServer.group_bytes([a, b]) == 10 * 1000 * 8
    assert FFTServer.group_bytes([d]) == 8192 * 4 + d.out_shape()[0] * 129 * 4
    with pytest.raises(ValueError):
        FFTRequest("fft1d", torch.zeros(10, dtype=torch.complex64)).key()
    with pytest.raises(ValueError):
        FFTRequest("fft3d", torch.zeros((2, 2), dtype=torch.complex64)).key()


def _mix(seed):
    import torch

    from reikna_b200.serve import FFTRequest

    rng = numpy.random.default_rng(seed)
    reqs = []
    for k in range(24):
        kind = ("fft1d", "fft1d", "fft1d", "fft2d", "spectrogram")[k % 5]
        if kind == "fft1d":
            n = int(rng.choice([64, 1000, 4096, 61, 3001, 2**17]))
            rows = int(rng.integers(1, 9))
            x = (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))).astype(numpy.complex64)
            reqs.append(FFTRequest(kind, torch.from_numpy(x).pin_memory(), inverse=int(rng.integers(0, 2))))
        elif kind == "fft2d":
            shape = [(64, 48), (128, 128), (100, 30)][k % 3]
            x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64)
            reqs.append(FFTRequest(kind, torch.from_numpy(x).pin_memory()))
        else:
            sig = rng.standard_normal(8192).astype(numpy.float32)
            reqs.append(FFTRequest(kind, torch.from_numpy(sig).pin_memory(), nfft=256, hop=64))
    return reqs


def _reference(r):
    x = r.data.numpy().astype(numpy.complex128 if r.kind != "spectrogram" else numpy.float64)
    if r.kind == "fft1d":
        return (numpy.fft.ifft if r.inverse else numpy.fft.fft)(x, axis=1), x.shape[1]
    if r.kind == "fft2d":
        return numpy.fft.fft2(x), x.size
    nf = (x.shape[0] - (r.nfft - r.hop)) // r.hop
    idx = numpy.arange(nf)[:, None] * r.hop + numpy.arange(r.nfft)[None, :]
    w = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(r.nfft) / (r.nfft - 1)))
    return numpy.abs(numpy.fft.rfft(x[idx] * w, axis=1)), r.nfft


@pytest.mark.gpu
@pytest.mark.parametrize("arrivals", ["burst", "poisson"])
def test_mix_equals_alone(arrivals):
    from reikna_b200.serve import FFTRequest, FFTServer

    reqs = _mix(31)
    offsets = None
    if arrivals == "poisson":
        offsets = numpy.cumsum(numpy.random.default_rng(32).exponential(200e-6, len(reqs))).tolist()
    srv = FFTServer(streams=3, depth=2, max_group_bytes=8 << 20)
    srv.run(reqs, offsets)
    assert all(r.done for r in reqs) and srv.completed == len(reqs)
    assert srv.groups < len(reqs) or arrivals == "poisson"
    for r in reqs:
        ref, n = _reference(r)
        got = r.result.numpy()
        assert rel_l2(got, ref) < fft_bound(numpy.complex64, n), r.key()
        # the same request served alone
        alone = FFTRequest(r.kind, r.data, inverse=r.inverse, nfft=r.nfft, hop=r.hop)
        one = FFTServer(streams=1, depth=1)
        one.run([alone])
        assert rel_l2(got, alone.result.numpy()) < fft_bound(numpy.complex64, n), r.key()
        assert r.finished >= r.launched >= r.arrival


@pytest.mark.gpu
def test_memory_budget_holds_groups_back():
    from reikna_b200.serve import FFTServer

    reqs = _mix(33)
    biggest = max(FFTServer.group_bytes([r]) for r in reqs)
    srv = FFTServer(streams=4, depth=4, memory_budget=biggest, max_group_bytes=1)
    peak = 0
    for r in reqs:
        srv.submit(r)
    while srv.pending:
        srv.step()
        peak = max(peak, srv._staged)
    assert peak <= max(biggest, srv.memory_budget)
    for r in reqs:
        ref, n = _reference(r)
        assert rel_l2(r.result.numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
def test_plain_per_call_matches_server():
    from reikna_b200.serve import serve_plain

    reqs = _mix(34)
    serve_plain(reqs)
    for r in reqs:
        ref, n = _reference(r)
        assert rel_l2(r.result.numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
def test_device_resident_requests():
    import torch

    from reikna_b200.serve import FFTRequest, FFTServer

    reqs = []
    for r in _mix(35):
        data = r.data.cuda()
        out = torch.empty(r.out_shape(), dtype=torch.float32 if r.kind == "spectrogram" else torch.complex64, device="cuda")
        reqs.append(FFTRequest(r.kind, data, inverse=r.inverse, nfft=r.nfft, hop=r.hop, out=out))
    srv = FFTServer(streams=2)
    srv.run(reqs)
    assert srv._staged == 0
    for r in reqs:
        host = FFTRequest(r.kind, r.data.cpu(), inverse=r.inverse, nfft=r.nfft, hop=r.hop)
        ref, n = _reference(host)
        assert r.result is r.out
        assert rel_l2(r.out.cpu().numpy(), ref) < fft_bound(numpy.complex64, n), r.key()
