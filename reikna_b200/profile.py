"""Run one FFT configuration a few times and report its per-pass times.

For profilers (``ncu ... python -m reikna_b200.profile ...``) and quick checks: the
computation is built and compiled once, run ``--steps`` times, then timed with CUDA
events around every pass (``rk_fft_profile``).

  python -m reikna_b200.profile --shape 256,256,256 [--axes 0,1,2] [--shift-scale]
      [--dtype complex64|complex128] [--flags N] [--steps 4] [--reps 200]
  python -m reikna_b200.profile --spectrogram 4194304 [--nfft 1024] [--hop 256]
      [--transposed] [--steps 4] [--reps 200]
"""

from __future__ import annotations

import argparse
import json
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--shape", help="comma-separated array shape")
    ap.add_argument("--spectrogram", type=int, default=0, help="signal length: profile the spectrogram instead")
    ap.add_argument("--nfft", type=int, default=1024)
    ap.add_argument("--hop", type=int, default=256)
    ap.add_argument("--transposed", action="store_true", help="spectrogram stored bins by frames")
    ap.add_argument("--axes", default=None, help="comma-separated transformed axes (default: all)")
    ap.add_argument("--dtype", default="complex64", choices=["complex64", "complex128"])
    ap.add_argument("--shift-scale", action="store_true", help="fused output fftshift and 1/N")
    ap.add_argument("--flags", type=int, default=0, help="plan flags (RK_FLAG_*)")
    ap.add_argument("--steps", type=int, default=4, help="untimed runs first")
    ap.add_argument("--reps", type=int, default=200, help="timed runs")
    args = ap.parse_args(argv)

    import torch

    from . import transformations as tr
    from .fft import FFT

    if args.spectrogram:
        return _spectrogram(args)
    if not args.shape:
        ap.error("--shape or --spectrogram is required")
    shape = tuple(int(v) for v in args.shape.split(","))
    axes = None if args.axes is None else tuple(int(v) for v in args.axes.split(","))
    dev = torch.device("cuda", 0)
    rdt = torch.float32 if args.dtype == "complex64" else torch.float64
    gen = torch.Generator(device=dev).manual_seed(1)
    x = torch.complex(torch.randn(shape, device=dev, dtype=rdt, generator=gen),
                      torch.randn(shape, device=dev, dtype=rdt, generator=gen))
    y = torch.empty_like(x)
    fft = FFT(x, axes=axes)
    if args.shift_scale:
        sh = tr.fftshift(x, axes=axes)
        sc = tr.mul_const(x, 1.0 / x.numel())
        fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
        fft.parameter.shifted.connect(sc, sc.input, result=sc.output)
    cc = fft.compile(dev, flags=args.flags)
    for _ in range(args.steps):
        cc(None, y, x)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.reps):
        cc(None, y, x)
    e.record()
    torch.cuda.synchronize()
    step_us = s.elapsed_time(e) / args.reps * 1e3
    out = {"shape": list(shape), "axes": axes, "dtype": args.dtype, "flags": args.flags, "us_per_step": step_us,
           "passes": _passes(cc, lambda: cc(None, y, x), args.reps)}
    print(json.dumps(out))
    return 0


def _passes(cc, call, reps: int) -> list:
    """Per-pass CUDA-event times of ``reps`` calls of a compiled FFT-based computation."""
    import torch

    plan = cc._runner.plan
    plan.profile(reps)
    for _ in range(reps):
        call()
    torch.cuda.synchronize()
    ms, calls = plan.profile_read()
    plan.profile(0)
    return [{"note": p["note"], "L": p["L"], "mode": p["mode"], "var": p["var"], "us": m / max(1, calls) * 1e3}
            for p, m in zip(plan.describe()["passes"], ms)]


def _spectrogram(args) -> int:
    import torch

    from .spectrogram import frames, spectrogram

    dev = torch.device("cuda", 0)
    n = args.spectrogram
    gen = torch.Generator(device=dev).manual_seed(1)
    x = torch.randn(n, device=dev, dtype=torch.float32, generator=gen)
    nf = frames(n, args.nfft, args.hop)
    nb = args.nfft // 2 + 1
    y = torch.empty((nb, nf) if args.transposed else (nf, nb), device=dev, dtype=torch.float32)
    cc = spectrogram(n, args.nfft, args.hop, transposed=args.transposed).compile(dev)
    for _ in range(args.steps):
        cc(None, y, x)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.reps):
        cc(None, y, x)
    e.record()
    torch.cuda.synchronize()
    out = {"spectrogram": n, "nfft": args.nfft, "hop": args.hop, "transposed": args.transposed,
           "us_per_step": s.elapsed_time(e) / args.reps * 1e3,
           "passes": _passes(cc, lambda: cc(None, y, x), args.reps)}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
