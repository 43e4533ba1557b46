"""The allocation-free 1-D FFT entry point (rk_fft1d_c64_noalloc) through the C ABI.

This entry point serves callers that may not allocate device memory while they run
a transform (a memory pool or arena that owns the device, a loop that must stay out
of the allocator, a host that lends only its own buffers): its intermediate buffer
and twiddle tables are static device arrays of the library.  The checks compare it
with the planned FFT (which allocates its temporaries) on two calls in a row, so a
second call that reused stale scratch contents would show up.  The file is named to
be collected last.
"""

import ctypes

import numpy
import pytest

from helpers import fft_bound, rel_l2

pytestmark = pytest.mark.gpu


def _noalloc(out, inp, n, batch, inverse):
    import torch

    from reikna_b200 import _native as N

    stream = torch.cuda.current_stream().cuda_stream
    return N.lib().rk_fft1d_c64_noalloc(
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(inp.data_ptr()), n, batch, inverse, ctypes.c_void_p(stream)
    )


def _planned(inp, inverse):
    import torch

    from reikna_b200.fft import FFT

    out = torch.empty_like(inp)
    FFT(inp, axes=(1,)).compile()(None, out, inp, inverse)
    return out


@pytest.mark.parametrize("n,batch", [(4096, 64), (2**16, 8), (2**20, 4)])
def test_noalloc_matches_planned_fft_twice(n, batch):
    import torch

    rng = numpy.random.default_rng(n + batch)
    dev = torch.device("cuda", 0)
    for call, inverse in enumerate((0, 1)):
        x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(numpy.complex64)
        t = torch.from_numpy(x).to(dev)
        out = torch.empty_like(t)
        assert _noalloc(out, t, n, batch, inverse) == 0
        ref = _planned(t, inverse)
        torch.cuda.synchronize()
        got, want = out.cpu().numpy(), ref.cpu().numpy()
        assert rel_l2(got, want) < fft_bound(numpy.complex64, n), (call, inverse)
        exact = numpy.fft.ifft(x.astype(numpy.complex128), axis=1) if inverse else numpy.fft.fft(x.astype(numpy.complex128), axis=1)
        assert rel_l2(got, exact) < fft_bound(numpy.complex64, n)


def test_noalloc_in_place():
    import torch

    n, batch = 8192, 16
    rng = numpy.random.default_rng(3)
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(numpy.complex64)
    t = torch.from_numpy(x).cuda()
    assert _noalloc(t, t, n, batch, 0) == 0
    torch.cuda.synchronize()
    assert rel_l2(t.cpu().numpy(), numpy.fft.fft(x.astype(numpy.complex128), axis=1)) < fft_bound(numpy.complex64, n)


def test_noalloc_rejects_oversize_and_bad_length():
    import torch

    from reikna_b200 import _native as N

    t = torch.zeros(8, dtype=torch.complex64, device="cuda")
    assert _noalloc(t, t, 2**20, 8, 0) == N.ERR_INVALID
    assert b"static scratch" in N.lib().rk_last_error()
    assert _noalloc(t, t, 3000, 1, 0) == N.ERR_INVALID
    assert b"power of two" in N.lib().rk_last_error()


def test_noalloc_repeat_after_other_size_is_identical_and_allocates_nothing():
    """A call repeated on the same input after a call of another size (which leaves
    different contents in the shared scratch) gives bit-identical output, and once
    every size has run once (set-up, tables, kernels loaded) further calls leave the
    device's free memory unchanged."""
    import torch

    rng = numpy.random.default_rng(11)
    dev = torch.device("cuda", 0)
    cases = [(2**16, 16), (4096, 512), (2**20, 2)]
    ins, outs = [], []
    for n, batch in cases:
        x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(numpy.complex64)
        ins.append(torch.from_numpy(x).to(dev))
        outs.append([torch.empty_like(ins[-1]) for _ in range(2)])
    for (n, batch), t, (o, _) in zip(cases, ins, outs):
        assert _noalloc(o, t, n, batch, 0) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for rep in range(3):
        for (n, batch), t, (_, o2) in zip(cases, ins, outs):
            assert _noalloc(o2, t, n, batch, rep % 2) == 0
            assert _noalloc(o2, t, n, batch, 0) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    for o, o2 in outs:
        assert torch.equal(o, o2)


def test_noalloc_rejects_foreign_memory():
    import torch

    from reikna_b200 import _native as N

    n, batch = 4096, 2
    t = torch.zeros((batch, n), dtype=torch.complex64, device="cuda")
    host = torch.zeros((batch, n), dtype=torch.complex64).pin_memory()
    assert _noalloc(t, host, n, batch, 0) == N.ERR_INVALID
    assert b"device memory of the current device" in N.lib().rk_last_error()
