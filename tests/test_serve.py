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


def _extremes(seed):
    """Requests at the serving stream's extremes: the largest prime length, the
    longest power of two with several rows, the largest 2-D transform and a full
    2^22-sample spectrogram at nfft 1024 / hop 256, mixed with small requests."""
    import torch

    from reikna_b200.serve import FFTRequest

    rng = numpy.random.default_rng(seed)

    def c64(shape):
        return torch.from_numpy((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64))

    reqs = [
        FFTRequest("fft1d", c64((3, 65521)).pin_memory()),
        FFTRequest("fft1d", c64((2, 65521)).pin_memory(), inverse=1),
        FFTRequest("fft1d", c64((4, 2**20)).pin_memory()),
        FFTRequest("fft2d", c64((2048, 2048)).pin_memory()),
        FFTRequest("fft1d", c64((256, 61)).pin_memory()),
        FFTRequest("fft1d", c64((5, 64)).pin_memory()),
    ]
    t = numpy.arange(2**22)
    sig = rng.standard_normal(2**22)
    for _ in range(8):
        sig += rng.uniform(0.1, 2) * numpy.sin(2 * numpy.pi * rng.uniform(0, 0.5) * t + rng.uniform(0, 2 * numpy.pi))
    reqs.append(FFTRequest("spectrogram", torch.from_numpy(sig.astype(numpy.float32)).pin_memory(), nfft=1024, hop=256))
    return reqs


@pytest.mark.gpu
def test_mix_extremes_equal_alone():
    from reikna_b200.serve import FFTRequest, FFTServer

    reqs = _extremes(36)
    srv = FFTServer(streams=3, depth=2)
    srv.run(reqs)
    assert all(r.status == "done" for r in reqs)
    for r in reqs:
        ref, n = _reference(r)
        got = r.result.numpy()
        assert rel_l2(got, ref) < fft_bound(numpy.complex64, n), r.key()
        alone = FFTRequest(r.kind, r.data, inverse=r.inverse, nfft=r.nfft, hop=r.hop)
        FFTServer(streams=1, depth=1).run([alone])
        assert rel_l2(got, alone.result.numpy()) < fft_bound(numpy.complex64, n), r.key()


# ---- failures stay with their requests ------------------------------------------------


def _host_req(rows, n, seed=0):
    import torch

    from reikna_b200.serve import FFTRequest

    rng = numpy.random.default_rng(seed)
    x = (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))).astype(numpy.complex64)
    return FFTRequest("fft1d", torch.from_numpy(x))


def test_oversize_request_rejected_at_submit():
    import torch

    from reikna_b200.serve import AdmissionError, FFTServer

    srv = FFTServer(torch.device("cuda", 0), memory_budget=64 << 10)
    small = srv.submit(_host_req(2, 1024))       # 16 KiB
    big = srv.submit(_host_req(16, 1024))        # 128 KiB > the whole budget
    assert small.status == "waiting" and not small.done
    assert big.status == "rejected" and big.done and isinstance(big.error, AdmissionError)
    assert srv.rejected == 1 and srv.pending == 1


def test_cancel_waiting_request():
    import torch

    from reikna_b200.serve import FFTServer

    srv = FFTServer(torch.device("cuda", 0))
    a, b, c = (srv.submit(_host_req(1, 256, s)) for s in range(3))
    assert srv.cancel(b)
    assert b.status == "cancelled" and b.done and srv.pending == 2
    assert not srv.cancel(b)
    assert [r.status for r in (a, c)] == ["waiting", "waiting"]


def test_plan_failure_fails_its_group_only(monkeypatch):
    """A class whose plan cannot be built fails its own requests and queues no GPU
    work; the other classes' requests stay queued."""
    import torch

    from reikna_b200 import serve

    def broken(key, rows):
        raise MemoryError("injected: plan allocation refused")

    monkeypatch.setattr(serve, "_computation", broken)
    srv = serve.FFTServer(torch.device("cuda", 0), streams=2, depth=1)
    bad = [srv.submit(_host_req(2, 4096, s)) for s in range(3)]
    srv.step()
    assert all(r.status == "failed" and r.done and isinstance(r.error, MemoryError) for r in bad)
    assert srv.failed == 3 and srv.pending == 0 and srv.streams is None  # nothing reached the GPU


@pytest.mark.gpu
def test_failures_isolated_on_gpu(monkeypatch):
    """Injected failures (a plan that cannot be compiled, a staging allocation that is
    refused) fail only their own groups; every other request is served correctly."""
    import torch

    from reikna_b200 import serve

    real = serve._computation

    def flaky(key, rows):
        if key[0] == "fft1d" and key[1] == 1000:
            raise MemoryError("injected: plan allocation refused")
        return real(key, rows)

    monkeypatch.setattr(serve, "_computation", flaky)
    srv = serve.FFTServer(streams=2, depth=2)
    real_alloc = srv._alloc

    def alloc(shape, dtype):
        if dtype == torch.complex64 and tuple(shape[1:]) == (96, 80):
            raise torch.cuda.OutOfMemoryError("injected: staging allocation refused")
        return real_alloc(shape, dtype)

    srv._alloc = alloc
    good = [_host_req(3, 4096, 1), _host_req(2, 61, 2), _host_req(7, 2**14, 3)]
    bad_plan = [_host_req(2, 1000, 4), _host_req(1, 1000, 5)]
    rng = numpy.random.default_rng(6)
    x2 = (rng.standard_normal((96, 80)) + 1j * rng.standard_normal((96, 80))).astype(numpy.complex64)
    bad_alloc = [serve.FFTRequest("fft2d", torch.from_numpy(x2))]
    reqs = good + bad_plan + bad_alloc
    srv.run(reqs)
    assert all(r.done for r in reqs)
    assert all(r.status == "failed" and isinstance(r.error, MemoryError) for r in bad_plan)
    assert bad_alloc[0].status == "failed" and isinstance(bad_alloc[0].error, torch.cuda.OutOfMemoryError)
    assert srv._staged == 0 and srv.failed == 3 and srv.completed == len(good)
    for r in good:
        assert r.status == "done"
        ref, n = _reference(r)
        assert rel_l2(r.result.numpy(), ref) < fft_bound(numpy.complex64, n)


@pytest.mark.gpu
@pytest.mark.parametrize("staged", [False, True])
def test_device_inputs_ordered_after_producer_stream(staged):
    """Device inputs still being written by a kernel queued on the submitter's side
    stream: the server waits for that stream (event recorded at submit) before it
    reads them, for direct (device output) and staged (host output) requests."""
    import torch

    from reikna_b200.serve import FFTRequest, FFTServer

    rng = numpy.random.default_rng(37)
    x = (rng.standard_normal((16, 4096)) + 1j * rng.standard_normal((16, 4096))).astype(numpy.complex64)
    src = torch.from_numpy(x).cuda()
    side = torch.cuda.Stream()
    srv = FFTServer(streams=2)
    with torch.cuda.stream(side):
        data = torch.zeros_like(src)
        torch.cuda._sleep(50_000_000)          # the producer is still queued when submitted
        data.copy_(src)
        out = None if staged else torch.empty_like(src)
        req = srv.submit(FFTRequest("fft1d", data, out=out))
    srv.drain()
    torch.cuda.synchronize()
    got = (req.result if staged else req.out).cpu().numpy()
    assert rel_l2(got, numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 4096)
