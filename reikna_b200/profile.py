"""Run one FFT configuration a few times and report its per-pass times.

For profilers (``ncu ... python -m reikna_b200.profile ...``) and quick checks: the
computation is built and compiled once, run ``--steps`` times, then timed with CUDA
events around every pass (``rk_fft_profile``).

  python -m reikna_b200.profile --shape 256,256,256 [--axes 0,1,2] [--shift-scale]
      [--dtype complex64|complex128] [--flags N] [--steps 4] [--reps 200]
"""

from __future__ import annotations

import argparse
import json
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--shape", required=True, help="comma-separated array shape")
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
    plan = cc._runner.plan
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.reps):
        cc(None, y, x)
    e.record()
    torch.cuda.synchronize()
    step_us = s.elapsed_time(e) / args.reps * 1e3
    plan.profile(args.reps)
    for _ in range(args.reps):
        cc(None, y, x)
    torch.cuda.synchronize()
    ms, calls = plan.profile_read()
    plan.profile(0)
    passes = plan.describe()["passes"]
    out = {"shape": list(shape), "axes": axes, "dtype": args.dtype, "flags": args.flags, "us_per_step": step_us,
           "passes": [{"note": p["note"], "L": p["L"], "mode": p["mode"], "var": p["var"],
                       "us": m / max(1, calls) * 1e3} for p, m in zip(passes, ms)]}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
