"""Bounded device waits: a dependency that can never complete makes the kernel give
up after the (runtime) wait limit and report it in the device status word; the
context stays usable and the next transform runs normally once the word is cleared.
The stall comes from a task list built on the host (the pass the task waits for has
no tiles), never from a fault."""

import ctypes
import time

import numpy
import pytest

from helpers import fft_bound, rel_l2


def test_wait_api_exported():
    from reikna_b200 import _native as N

    for name in ("rk_set_wait_limit", "rk_get_wait_limit", "rk_stream_check", "rk_selftest_stalled_wait"):
        assert hasattr(N.lib(), name)


@pytest.mark.gpu
def test_stalled_dependency_times_out_then_recovers():
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    N.device_status(clear=True)
    default = N.wait_limit()
    assert default >= 10**9
    N.set_wait_limit(2_000_000)          # about 1 ms of SM clock
    try:
        assert N.wait_limit() == 2_000_000
        stream = torch.cuda.current_stream().cuda_stream
        t0 = time.perf_counter()
        rc = N.lib().rk_selftest_stalled_wait(ctypes.c_void_p(stream))
        dt = time.perf_counter() - t0
        assert rc == N.ERR_DEVICE
        assert b"bounded wait ran out" in N.lib().rk_last_error()
        assert dt < 0.5, dt                       # gave up after ~1 ms, not the default ~1 s
        word = N.device_status(clear=True)
        assert word & N.STATUS_TIMEOUT
        assert N.device_status() == 0
    finally:
        N.set_wait_limit(default)
    # the context is intact: a normal transform runs and leaves the word clear
    rng = numpy.random.default_rng(5)
    x = (rng.standard_normal((8, 4096)) + 1j * rng.standard_normal((8, 4096))).astype(numpy.complex64)
    t = torch.from_numpy(x).cuda()
    out = torch.empty_like(t)
    FFT(t, axes=(1,)).compile()(None, out, t)
    N.stream_check(torch.cuda.current_stream().cuda_stream)
    assert rel_l2(out.cpu().numpy(), numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, 4096)
    assert N.device_status() == 0


@pytest.mark.gpu
def test_wait_limit_rejects_tiny_values():
    from reikna_b200 import _native as N

    with pytest.raises(ValueError):
        N.set_wait_limit(10)
