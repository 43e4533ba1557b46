#!/usr/bin/env python
"""Benchmark of the FFT hot path on B200.

Workload (the configuration the headline metric is quoted on): 3-D C2C FFT over all
axes of a 256 x 256 x 256 complex64 array with a fused output fftshift and 1/N
scaling transformation.  One step = one forward transform of one array resident in
HBM; inputs are 134 MB each (larger than the 126 MB L2) and three input/output sets
rotate between steps.  Consecutive steps are independent and rotate over three
streams (one compiled plan and buffer set each), so a step's first pass overlaps the
earlier steps' second passes; ``ms_per_step_one_stream`` reports the same steps run
back to back on one stream, and the roofline's per-kernel durations come from CUDA
events around every launch in a separate single-stream loop.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl own|reference]

Metric: algorithmic HBM throughput in GB/s, B_alg = P_min * (bytes_in + bytes_out)
with P_min = ceil(log2(2^24) / log2(2^14)) = 2, i.e. 536,870,912 bytes per step.
``e2e`` times the same call through the public API with pinned host buffers and the
host<->device copies inside the timed region.  ``--impl reference`` times the CPU
restatement of reikna's FFT (oracle/) on the host cores instead.
Multi-GPU: one independent replica per GPU (no data-path collective; the transform
does not need to shard), value = all replicas' bytes / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

SHAPE = (256, 256, 256)
NTOT = SHAPE[0] * SHAPE[1] * SHAPE[2]
ELEM = 8
ARRAY_BYTES = NTOT * ELEM
P_MIN = 2
B_ALG = P_MIN * 2 * ARRAY_BYTES
# streams the headline loop rotates consecutive steps over (measured per step on one
# B200: 1 stream 154 us, 2: 134, 3: 120, 4: 124.5)
LANES = 3
FLOP = 5 * NTOT * math.log2(NTOT)
METRIC = "C2C FFT GB/s vs HBM peak, plain vs batched/TC-split at stated err; serve p99 ms"
CONFIG = {
    "workload": "fft3d_256^3_complex64_fftshift_scale",
    "shape": list(SHAPE),
    "dtype": "complex64",
    "axes": [0, 1, 2],
    "transformations": ["fftshift (output)", "mul_const 1/N (output)"],
    "bytes_per_step_algorithmic": B_ALG,
    "l2": "inputs larger than L2 (134 MB each), three buffer sets rotate (one per stream)",
}


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:  # noqa: BLE001
            pass
    return 6650.0, "fallback"


def traffic_from_profiles(kernel_note: str):
    """DRAM bytes per launch recorded by an ncu capture summary under profiles/ (copied
    from that capture, not measured in this run); returns (bytes, file) or (None, None)."""
    for f in sorted((ROOT / "profiles").glob("*.md")) + sorted((ROOT / "profiles").glob("*.txt")):
        txt = f.read_text(errors="replace")
        m = re.search(rf"traffic\[{re.escape(kernel_note)}\]\s*=\s*([0-9.eE+]+)", txt)
        if m:
            return float(m.group(1)), f"profiles/{f.name}"
    return None, None


class Clocks:
    """SM clock and throttle-reason samples taken by a background thread through NVML
    (read-only queries) every ``period`` seconds while the block runs.  The GPU is
    found by its PCI bus id, so CUDA_VISIBLE_DEVICES remapping does not matter.
    ``hold(seconds)`` keeps sampling a little longer (a workload whose timed steps
    take milliseconds is kept running around them, see ``soak`` in the callers)."""

    REASONS = (
        ("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
        ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
        ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
        ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
    )

    def __init__(self, device_index: int, period: float = 0.01):
        self.device_index = device_index
        self.period = period
        self.rows = []
        self.error = None
        self._stop = None
        self._thread = None

    def _handle(self, nv):
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.device_index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:  # noqa: BLE001 - fall back to the index
            return nv.nvmlDeviceGetHandleByIndex(self.device_index)

    def _run(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            try:
                h = self._handle(nv)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                bits = [(name, getattr(nv, attr, 0)) for name, attr in self.REASONS]
                while not self._stop.is_set():
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    why = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    util = nv.nvmlDeviceGetUtilizationRates(h).gpu
                    self.rows.append((sm, mx, why, util, [n for n, bit in bits if why & bit]))
                    self._stop.wait(self.period)
            finally:
                nv.nvmlShutdown()
        except Exception as e:  # noqa: BLE001 - no NVML: the line says so
            self.error = f"{type(e).__name__}: {e}"

    def __enter__(self):
        import threading

        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thread.join(timeout=5)

    def summary(self) -> dict:
        rows = list(self.rows)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0,
                    "error": self.error}
        # samples under load: GPU utilisation above zero in NVML's last sampling window
        busy = [r for r in rows if r[3] > 0] or rows
        return {
            "sm_mhz": statistics.median(r[0] for r in busy),
            "sm_max_mhz": max(r[1] for r in rows),
            "reasons": sorted({n for r in busy for n in r[4]}),
            "samples": len(rows),
            "samples_under_load": len(busy),
            "source": "NVML, background thread, 10 ms period",
        }


def soak(fn, seconds: float) -> None:
    """Keep the GPU on the workload for ``seconds`` (untimed) so that the clock
    sampler sees it under load around a short timed region."""
    import torch

    t_end = time.perf_counter() + seconds
    while time.perf_counter() < t_end:
        fn()
        torch.cuda.synchronize()


def cpu_baseline(x_host, seconds: float = 12.0) -> dict:
    """The reikna-algorithm CPU oracle on this host, full workload per sample."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    plan = oracle.Plan(SHAPE, (0, 1, 2))
    out = x_host.copy()
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < 2 or (time.perf_counter() < t_end and len(times) < 50):
        t0 = time.perf_counter()
        plan.shifted(x_host, scale=1.0 / NTOT, threads=threads, out=out)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times[1:]) if len(times) > 2 else times[-1]
    return {
        "value": B_ALG / t / 1e9,
        "unit": "GB/s",
        "cores": threads,
        "kind": "port",
        "sample": f"full 256^3 complex64 FFT + fftshift + 1/N per sample, median of {len(times) - 1} after 1 warm-up",
        "ms_per_step": t * 1e3,
    }


def run_reference(args, rank: int, world: int) -> int:
    if rank != 0:
        return 0
    import numpy

    from oracle import oracle

    rng = numpy.random.default_rng(2)
    x = (rng.standard_normal(SHAPE, numpy.float32) + 1j * rng.standard_normal(SHAPE, numpy.float32)).astype(numpy.complex64)
    threads = os.cpu_count() or 1
    plan = oracle.Plan(SHAPE, (0, 1, 2))
    out = numpy.empty_like(x)
    tw = time.perf_counter()
    for _ in range(args.warmup):
        plan.shifted(x, scale=1.0 / NTOT, threads=threads, out=out)
    per = (time.perf_counter() - tw) / max(1, args.warmup)
    # a step is one full transform on the host cores (about 0.2 s); the run is held to
    # about two minutes, so at most that many steps of the K requested are timed
    steps = max(1, min(args.steps, int(120.0 / max(per, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        plan.shifted(x, scale=1.0 / NTOT, threads=threads, out=out)
    t = (time.perf_counter() - t0) / steps
    value = B_ALG / t / 1e9
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "steps_timed": steps,
        "warmup": args.warmup,
        "ms_per_step": t * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": CONFIG,
        "cpu_baseline": {
            "value": value,
            "unit": "GB/s",
            "cores": threads,
            "kind": "port",
            "sample": "full 256^3 complex64 FFT + fftshift + 1/N per step (C restatement of reikna's algorithm, OpenMP)",
        },
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gflops": FLOP / t / 1e9,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_own(args, rank: int, world: int, local_rank: int) -> int:
    import numpy
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    gen = torch.Generator(device=dev).manual_seed(1234 + rank)
    xs = [torch.complex(torch.randn(SHAPE, device=dev, generator=gen), torch.randn(SHAPE, device=dev, generator=gen))
          for _ in range(LANES)]
    outs = [torch.empty_like(xs[0]) for _ in range(LANES)]

    def build():
        fft = FFT(xs[0])
        sh = tr.fftshift(xs[0])
        sc = tr.mul_const(xs[0], 1.0 / NTOT)
        fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
        fft.parameter.shifted.connect(sc, sc.input, result=sc.output)
        return fft.compile(dev)

    # consecutive steps are independent transforms of rotating buffer sets: step k runs
    # on stream k % LANES with its own compiled plan (each plan owns the intermediate
    # between its two passes), so one step's plane pass overlaps the previous steps'
    # lane passes
    comps = [build() for _ in range(LANES)]
    comp = comps[0]
    plan = comp._runner.plan
    launches = plan.launches
    passes = plan.describe()["passes"]

    stream = torch.cuda.current_stream(dev)
    lanes = [torch.cuda.Stream(dev) for _ in range(LANES)]
    for k in range(args.warmup):
        comps[k % LANES](lanes[k % LANES], outs[k % LANES], xs[k % LANES])
    torch.cuda.synchronize(dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def round_of_steps():
        for k in range(LANES * 8):
            comps[k % LANES](lanes[k % LANES], outs[k % LANES], xs[k % LANES])

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        soak(round_of_steps, 0.5)
        barrier()
        torch.cuda.synchronize(dev)
        start.record(stream)
        for s in lanes:
            s.wait_stream(stream)
        for k in range(args.steps):
            comps[k % LANES](lanes[k % LANES], outs[k % LANES], xs[k % LANES])
        for s in lanes:
            stream.wait_stream(s)
        end.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        soak(round_of_steps, 0.2)
    ms = start.elapsed_time(end)
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * B_ALG * args.steps / (ms / 1e3) / 1e9

    # the same steps one after another on one stream (no overlap), and the per-pass
    # kernel durations from CUDA events around every launch (a separate timed loop:
    # the events between launches cost about 10 us a step)
    serial_steps = max(3, min(args.steps, 500))
    s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    s1.record(stream)
    for k in range(serial_steps):
        comp(stream, outs[k % 2], xs[k % 2])
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_serial = s1.elapsed_time(e1) / serial_steps
    plan.profile(serial_steps)
    for k in range(serial_steps):
        comp(stream, outs[k % 2], xs[k % 2])
    torch.cuda.synchronize(dev)
    pass_ms, calls = plan.profile_read()
    plan.profile(0)
    if dist is not None:
        t = torch.tensor([ms_serial], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_serial = float(t.item())

    # end to end through the public API with pinned host buffers: every step copies
    # its input up, transforms it and copies the result down; consecutive steps are
    # pipelined over an upload, a compute and a download stream (two buffer sets),
    # so the link carries both directions at once
    h_in = xs[0].cpu().pin_memory()
    h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    d_in = [torch.empty_like(xs[0]) for _ in range(2)]
    d_out = [torch.empty_like(xs[0]) for _ in range(2)]
    up_s, cp_s, dn_s = (torch.cuda.Stream(dev) for _ in range(3))
    up_ev = [torch.cuda.Event() for _ in range(2)]
    cp_ev = [torch.cuda.Event() for _ in range(2)]
    dn_ev = [torch.cuda.Event() for _ in range(2)]
    e2e_steps = max(2, min(args.steps, 20))

    def e2e_step(k):
        b = k % 2
        with torch.cuda.stream(up_s):
            if k >= 2:
                up_s.wait_event(cp_ev[b])  # the transform of step k-2 has read d_in[b]
            d_in[b].copy_(h_in, non_blocking=True)
            up_ev[b].record(up_s)
        cp_s.wait_event(up_ev[b])
        if k >= 2:
            cp_s.wait_event(dn_ev[b])      # d_out[b] of step k-2 is downloaded
        comp(cp_s, d_out[b], d_in[b])
        cp_ev[b].record(cp_s)
        with torch.cuda.stream(dn_s):
            dn_s.wait_event(cp_ev[b])
            h_out[b].copy_(d_out[b], non_blocking=True)
            dn_ev[b].record(dn_s)

    for k in range(3):
        e2e_step(k)
    torch.cuda.synchronize(dev)
    barrier()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(up_s)
    cp_s.wait_event(s2)
    dn_s.wait_event(s2)
    for k in range(e2e_steps):
        e2e_step(k)
    e2.record(dn_s)
    torch.cuda.synchronize(dev)
    ms_e2e = s2.elapsed_time(e2)
    h_last = h_out[(e2e_steps - 1) % 2]
    if dist is not None:
        t = torch.tensor([ms_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
        barrier()
        dist.destroy_process_group()

    if rank != 0:
        return 0

    # accuracy of the timed computation against the FP64 reference (outside timing)
    x_host = xs[0].cpu().numpy()
    y = h_last.numpy()
    ref = numpy.fft.fftshift(numpy.fft.fftn(x_host.astype(numpy.complex128))) / NTOT
    err = float(numpy.linalg.norm((y - ref).ravel()) / numpy.linalg.norm(ref.ravel()))

    peak, peak_kind = peaks()
    per_launch = [m / max(1, calls) for m in pass_ms]
    dom = max(range(len(per_launch)), key=lambda i: per_launch[i])
    dom_bytes = 2 * ARRAY_BYTES  # each pass reads and writes the whole array once
    achieved = dom_bytes / (per_launch[dom] / 1e3) / 1e9
    traffic, traffic_src = traffic_from_profiles(passes[dom]["note"] + f"/L{passes[dom]['L']}/{passes[dom]['mode']}")
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(CONFIG, parallelism=f"replicas{world}"),
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, copied from {traffic_src}"
            if traffic_src else None,
            "kernel": passes[dom]["note"] + f" L={passes[dom]['L']} {passes[dom]['mode']}",
            "bytes_per_launch_algorithmic": dom_bytes,
            "ms_per_launch": per_launch[dom],
            "peak_kind": peak_kind,
        },
        "hbm_frac_step": (B_ALG / (ms / args.steps / 1e3) / 1e9) / peak,
        "ms_per_step_one_stream": ms_serial,
        "overlap": f"consecutive steps rotate over {LANES} streams with one compiled plan and buffer set each",
        "pass_ms": per_launch,
        "passes": [f"{p['note']} L={p['L']} {p['mode']}" for p in passes],
        "gflops": world * FLOP * args.steps / (ms / 1e3) / 1e9,
        "rel_l2_vs_fp64": err,
        "e2e": {
            "value": world * B_ALG * e2e_steps / (ms_e2e / 1e3) / 1e9,
            "unit": "GB/s",
            "h2d_bytes_per_step": ARRAY_BYTES,
            "d2h_bytes_per_step": ARRAY_BYTES,
            "ms_per_step": ms_e2e / e2e_steps,
            "pipelining": "upload, transform and download of consecutive steps overlap on three streams",
        },
        "gpu_launches": launches * args.steps,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_configs:
        line["configs"] = measure_configs(dev, args)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(x_host)
    print(json.dumps(line), flush=True)
    return 0


# --- the other configurations, measured beside the headline ----------------------------


def _rel(a, b) -> float:
    import numpy

    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    return float(numpy.linalg.norm((a - b).ravel()) / numpy.linalg.norm(b.ravel()))


def _events_ms(fn, reps: int) -> float:
    import torch

    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s0.record()
    for _ in range(reps):
        fn()
    s1.record()
    torch.cuda.synchronize()
    return s0.elapsed_time(s1) / reps


def measure_c1(dev, warmup: int) -> dict:
    """Plain 1-D C2C: 64 x 4096 complex64 along the last axis, forward then inverse.
    80 buffer sets rotate (160 MB of inputs, more than L2).  Per-call: one forward and
    one inverse call through the public API per set; graph: the same 160 calls
    captured once in a CUDA graph and replayed."""
    import numpy
    import torch

    from reikna_b200.fft import FFT

    nset, shape = 80, (64, 4096)
    rng = numpy.random.default_rng(1)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64)
    xs = [torch.from_numpy(x).to(dev) for _ in range(nset)]
    ys = [torch.empty_like(xs[0]) for _ in range(nset)]
    zs = [torch.empty_like(xs[0]) for _ in range(nset)]
    cc = FFT(xs[0], axes=(1,)).compile(dev)

    def pairs():
        for k in range(nset):
            cc(None, ys[k], xs[k], 0)
            cc(None, zs[k], ys[k], 1)

    for _ in range(max(3, warmup)):
        pairs()
    t0 = time.perf_counter()
    ms_calls = _events_ms(pairs, 5) / nset
    host_us = (time.perf_counter() - t0) / (5 * nset) * 1e6
    err_f = _rel(ys[0].cpu().numpy(), numpy.fft.fft(x.astype(numpy.complex128), axis=1))
    err_rt = _rel(zs[0].cpu().numpy(), x)
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        pairs()
    side.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        pairs()
    for _ in range(3):
        g.replay()
    ms_graph = _events_ms(g.replay, 10) / nset
    b_pair = 2 * 2 * x.nbytes            # forward + inverse, each reads and writes the array
    peak, _ = peaks()

    def entry(ms):
        gbs = b_pair / (ms / 1e3) / 1e9
        return {"us_per_pair": ms * 1e3, "gbs": gbs, "hbm_frac": gbs / peak}

    return {
        "workload": "64x4096 complex64, axis 1, forward + inverse (round trip)",
        "bytes_algorithmic_per_pair": b_pair,
        "per_call": dict(entry(ms_calls), host_us_per_pair=host_us),
        "graph": entry(ms_graph),
        "rel_l2_vs_fp64": err_f,
        "round_trip_rel_l2": err_rt,
        "launches_per_pair": 2 * cc.launches,
        "l2": f"{nset} buffer sets rotate ({nset * x.nbytes >> 20} MiB of inputs)",
    }


def measure_c2b(dev, warmup: int) -> dict:
    """3-D FP64 path: 128^3 complex128 over all axes with fused fftshift and 1/N; four
    buffer sets rotate (134 MB of inputs, more than L2)."""
    import numpy
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.fft import FFT

    shape, nset = (128, 128, 128), 4
    n = 128**3
    rng = numpy.random.default_rng(3)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    xs = [torch.from_numpy(x).to(dev) for _ in range(nset)]
    ys = [torch.empty_like(xs[0]) for _ in range(nset)]
    fft = FFT(xs[0])
    sh = tr.fftshift(xs[0])
    sc = tr.mul_const(xs[0], 1.0 / n)
    fft.parameter.output.connect(sh, sh.input, shifted=sh.output)
    fft.parameter.shifted.connect(sc, sc.input, result=sc.output)
    cc = fft.compile(dev)
    state = {"k": 0}

    def step():
        k = state["k"] % nset
        cc(None, ys[k], xs[k])
        state["k"] += 1

    for _ in range(max(3, warmup)):
        step()
    ms = _events_ms(step, 200)
    cc(None, ys[0], xs[0])
    err = _rel(ys[0].cpu().numpy(), numpy.fft.fftshift(numpy.fft.fftn(x)) / n)
    b_alg = 2 * 2 * x.nbytes              # P_min = 2 (2^21 points, 2^13 complex128 an SM)
    peak, _ = peaks()
    gbs = b_alg / (ms / 1e3) / 1e9
    return {"workload": "128^3 complex128, all axes, fftshift + 1/N (output)", "us_per_step": ms * 1e3,
            "bytes_algorithmic": b_alg, "gbs": gbs, "hbm_frac": gbs / peak, "rel_l2_vs_fp64": err,
            "bound": 1e-14 * 21, "passes": [p["note"] for p in cc._runner.plan.describe()["passes"]],
            "l2": f"{nset} buffer sets rotate"}


def measure_configs(dev, args) -> dict:
    """C1, C2b, C3, C4 and C5 in compact form for the default line (each entry: error
    against numpy FP64, device time, algorithmic GB/s and fraction of measured HBM)."""
    import torch

    peak, peak_kind = peaks()
    out = {"peak_gbs": peak, "peak_kind": peak_kind}
    t0 = time.perf_counter()
    steps = max(20, min(args.steps, 200))
    try:
        out["C1"] = measure_c1(dev, args.warmup)
        out["C2b"] = measure_c2b(dev, args.warmup)
        res, b_alg = measure_batch(dev, steps, args.warmup, modes=("graph_par", "persistent", "auto"))
        for v in res.values():
            v["hbm_frac"] = v["gbs"] / peak
        out["C3"] = {"workload": "batch 1000x3001 (Bluestein) + 1000x1000 + r2c 1000x1000", "bytes_algorithmic": b_alg,
                     "modes": res, "speedup_vs_plain": res["plain_per_call"]["us"] / res["auto"]["us"]}
        prec, b_alg = measure_precision(dev, steps, args.warmup)
        out["C4"] = {"workload": "16384x1024 complex64, axis 1", "bytes_algorithmic": b_alg, "results": prec}
        torch.cuda.empty_cache()
        out["C5"] = {
            "device_data": measure_serve(dev, args.serve_sample, "device", 4, 0.7, clocks=False),
            "host_data": measure_serve(dev, args.serve_sample, "host", 4, 0.7, clocks=False),
        }
    except Exception as e:  # noqa: BLE001 - the headline stands on its own
        out["error"] = f"{type(e).__name__}: {e}"
    out["seconds"] = time.perf_counter() - t0
    return out


# --- serving stream ---------------------------------------------------------------


def _primes_log_spaced(count: int = 16, lo: int = 61, hi: int = 65521) -> list[int]:
    """``count`` primes spread log-uniformly over [lo, hi] (the largest prime at or
    below each log-spaced target)."""
    import numpy

    sieve = numpy.ones(hi + 1, bool)
    sieve[:2] = False
    for k in range(2, int(hi**0.5) + 1):
        if sieve[k]:
            sieve[k * k :: k] = False
    primes = numpy.nonzero(sieve)[0]
    out = []
    for t in numpy.geomspace(lo, hi, count):
        out.append(int(primes[numpy.searchsorted(primes, t, side="right") - 1]))
    return sorted(set(out))


def _p_min(m: int, c_log: int = 14) -> int:
    import math

    return max(1, math.ceil(math.log2(max(m, 2)) / c_log))


def _bpow2(n: int) -> int:
    return 1 << (n - 1).bit_length()


def serve_stream(n: int, seed: int, dev, on_device: bool = False):
    """Synthetic request stream (seeded): 60% 1-D C2C with N uniform over the powers of
    two 2^6..2^20 and 16 log-spaced primes in [61, 65521], rows U{1..256}; 20% 2-D C2C
    with each side a power of two in 2^6..2^11; 20% spectrograms of a 2^22-sample
    float32 signal (N(0,1) plus 8 sinusoids), Hann window 1024, hop 256.  Inputs are
    views of shared pinned pools (their contents do not change the work); results go
    to shared pinned output pools.  Returns (requests, algorithmic bytes per request)."""
    import numpy
    import torch

    from reikna_b200.serve import FFTRequest
    from reikna_b200.spectrogram import frames

    rng = numpy.random.default_rng(seed)
    lengths = [2**k for k in range(6, 21)] + _primes_log_spaced()
    cap = 2**20 * 256
    gen = torch.Generator(device=dev).manual_seed(seed)
    pool = torch.complex(torch.randn(cap, device=dev, generator=gen), torch.randn(cap, device=dev, generator=gen))
    if on_device:
        out_pool = torch.empty(cap, dtype=torch.complex64, device=dev)
    else:
        pool = pool.cpu().pin_memory()
        out_pool = torch.empty(cap, dtype=torch.complex64).pin_memory()
    slen, nfft, hop = 2**22, 1024, 256
    t = numpy.arange(slen)
    sig = rng.standard_normal(slen)
    for _ in range(8):
        sig += rng.uniform(0.1, 2) * numpy.sin(2 * numpy.pi * rng.uniform(0, 0.5) * t + rng.uniform(0, 2 * numpy.pi))
    sig_t = torch.from_numpy(sig.astype(numpy.float32))
    spec_out = torch.empty((frames(slen, nfft, hop), nfft // 2 + 1), dtype=torch.float32)
    sig_t, spec_out = (sig_t.to(dev), spec_out.to(dev)) if on_device else (sig_t.pin_memory(), spec_out.pin_memory())
    reqs, nbytes = [], []
    for _ in range(n):
        u = rng.uniform()
        if u < 0.6:
            ln = int(rng.choice(lengths))
            rows = int(rng.integers(1, 257))
            data = pool[: rows * ln].view(rows, ln)
            reqs.append(FFTRequest("fft1d", data, out=out_pool[: rows * ln].view(rows, ln)))
            m = ln if ln & (ln - 1) == 0 else 2 * _bpow2(ln)
            nbytes.append(_p_min(m) * 2 * rows * ln * 8)
        elif u < 0.8:
            n1, n2 = (2 ** int(rng.integers(6, 12)) for _ in range(2))
            data = pool[: n1 * n2].view(n1, n2)
            reqs.append(FFTRequest("fft2d", data, out=out_pool[: n1 * n2].view(n1, n2)))
            nbytes.append(_p_min(n1 * n2) * 2 * n1 * n2 * 8)
        else:
            reqs.append(FFTRequest("spectrogram", sig_t, nfft=nfft, hop=hop, out=spec_out))
            nbytes.append(_p_min(nfft) * (slen * 4 + spec_out.numel() * 4))
    return reqs, nbytes


def _reset(reqs):
    for r in reqs:
        r.done = False
        r.result = None
        r.arrival = r.launched = r.finished = 0.0


def _lat_ms(reqs) -> dict:
    import numpy

    lat = numpy.array([r.latency for r in reqs]) * 1e3
    return {"p50": float(numpy.percentile(lat, 50)), "p99": float(numpy.percentile(lat, 99)), "mean": float(lat.mean())}


def measure_serve(dev, n_requests: int, data: str, streams: int, load: float, clocks: bool = True) -> dict:
    """The serving stream's first ``n_requests`` requests through the continuous-batching
    server and through per-call plain execution: a burst (all arrive at t = 0) and a
    Poisson stream at ``load`` times the served burst rate.  Every result is checked
    against numpy FP64 on a seeded subset after the timed runs."""
    import collections

    import numpy
    import torch

    from reikna_b200.serve import FFTServer, serve_plain

    on_device = data == "device"
    reqs, nbytes = serve_stream(n_requests, 9, dev, on_device)
    total = float(sum(nbytes))
    srv = FFTServer(dev, memory_budget=40 << 30, streams=streams, depth=2)
    plain_cache = collections.OrderedDict()
    # warm pass of each arm: plans compiled and resident
    t_prep = time.perf_counter()
    srv.prepare(reqs)
    t_prep = time.perf_counter() - t_prep
    srv.run(reqs)
    _reset(reqs)
    torch.cuda.empty_cache()
    serve_plain(reqs, dev, cache=plain_cache)
    _reset(reqs)
    torch.cuda.synchronize(dev)
    warm_compiles = srv.plans.compiles
    with Clocks(dev.index) as clk:
        t_srv = srv.run(reqs)
        _reset(reqs)
        t_plain = serve_plain(reqs, dev, cache=plain_cache)
        _reset(reqs)
        rate = load * len(reqs) / t_srv
        offs = numpy.cumsum(numpy.random.default_rng(10).exponential(1.0 / rate, len(reqs))).tolist()
        t_srv_p = srv.run(reqs, offs)
        lat_srv = _lat_ms(reqs)
        _reset(reqs)
        t_plain_p = serve_plain(reqs, dev, offsets=offs, cache=plain_cache)
        lat_plain = _lat_ms(reqs)
    # the floor any batching of these requests meets: every request's transform
    # enqueued back to back on one stream from device-resident data, no host round
    # trips and no copies (device time of the kernels themselves, CUDA events)
    floor_s = None
    if on_device:
        calls = []
        for r in reqs:
            k = (r.key(), tuple(r.data.shape))
            cc = plain_cache[k]
            y = r.out if r.out is not None else None
            calls.append((cc, r, y))

        def enqueue_all():
            for cc, r, y in calls:
                if r.kind == "spectrogram":
                    cc(None, y, r.data)
                else:
                    cc(None, y, r.data, int(r.inverse))

        enqueue_all()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        enqueue_all()
        e1.record()
        torch.cuda.synchronize(dev)
        floor_s = e0.elapsed_time(e1) / 1e3
    # served results against numpy FP64 (a few requests of each kind; outputs of the
    # stream share pools, so each checked request is served again on its own buffers)
    errs = {}
    for r in [r for r in reqs if r.kind == "fft1d"][:2] + [r for r in reqs if r.kind == "fft2d"][:1] + \
            [r for r in reqs if r.kind == "spectrogram"][:1]:
        from reikna_b200.serve import FFTRequest

        one = FFTRequest(r.kind, r.data, inverse=r.inverse, nfft=r.nfft, hop=r.hop)
        srv.run([one])
        got = one.result.cpu().numpy() if hasattr(one.result, "cpu") else one.result.numpy()
        x = r.data.cpu().numpy()
        if r.kind == "fft1d":
            ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
        elif r.kind == "fft2d":
            ref = numpy.fft.fft2(x.astype(numpy.complex128))
        else:
            nf = got.shape[0]
            idx = numpy.arange(nf)[:, None] * r.hop + numpy.arange(r.nfft)[None, :]
            w = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(r.nfft) / (r.nfft - 1)))
            ref = numpy.abs(numpy.fft.rfft(x.astype(numpy.float64)[idx] * w, axis=1))
        errs[f"{r.kind}{list(r.data.shape)}"] = float(numpy.linalg.norm((got - ref).ravel()) / numpy.linalg.norm(ref.ravel()))
    h2d = sum(r.in_bytes() for r in reqs)
    d2h = sum(int(numpy.prod(r.out_shape())) * (4 if r.kind == "spectrogram" else 8) for r in reqs)
    kinds = collections.Counter(r.kind for r in reqs)
    return {
        "requests": len(reqs),
        "of_stream": "first requests of the seeded 100k-request stream (same generator)",
        "mix": dict(kinds),
        "data": data,
        "streams": streams,
        "bytes_algorithmic": total,
        "served": {"s": t_srv, "req_per_s": len(reqs) / t_srv, "gbs": total / t_srv / 1e9},
        "plain": {"s": t_plain, "req_per_s": len(reqs) / t_plain, "gbs": total / t_plain / 1e9},
        "speedup_vs_plain": t_plain / t_srv,
        "device_floor": None if floor_s is None else {
            "s": floor_s, "note": "every request's kernels back to back on one stream, no host round trips",
            "max_speedup_vs_plain": t_plain / floor_s, "served_vs_floor": t_srv / floor_s},
        "poisson": {"rate_req_per_s": rate, "load_vs_served_capacity": load, "served_latency_ms": lat_srv,
                    "plain_latency_ms": lat_plain, "served_s": t_srv_p, "plain_s": t_plain_p},
        "groups": srv.groups,
        "plans": {"prepared": warm_compiles, "prepare_s": t_prep,
                  "compiled_while_timed": srv.plans.compiles - warm_compiles, "evictions": srv.plans.evictions,
                  "resident_bytes": srv.plans.bytes, "plain_cache_plans": len(plain_cache)},
        "h2d_bytes": 0 if on_device else h2d,
        "d2h_bytes": 0 if on_device else d2h,
        "rel_l2_vs_fp64": errs,
        "clocks": clk.summary() if clocks else None,
    }


def run_serve(args, rank: int, world: int, local_rank: int) -> int:
    """Serving stream: continuous-batching server against per-call plain execution."""
    import torch

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    m = measure_serve(dev, args.requests, args.serve_data, args.streams, args.load)
    t_srv = m["served"]["s"]
    total = m["bytes_algorithmic"]
    line = {
        "metric": METRIC,
        "value": total / t_srv / 1e9,
        "unit": "GB/s",
        "n_gpus": 1,
        "steps": 1,
        "warmup": 1,
        "ms_per_step": t_srv * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": "serve_stream",
            "requests": m["requests"],
            "mix": m["mix"],
            "memory_budget_bytes": 40 << 30,
            "streams": args.streams,
            "data": args.serve_data,
            "note": "value = algorithmic bytes of all requests / wall time of a burst (all arrive at t=0); "
            + ("inputs and outputs in device memory" if args.serve_data == "device"
               else "host pinned inputs and outputs, copies included"),
        },
        "req_per_s": m["served"]["req_per_s"],
        "plain": {"value": m["plain"]["gbs"], "req_per_s": m["plain"]["req_per_s"], "s": m["plain"]["s"]},
        "speedup_vs_plain": m["speedup_vs_plain"],
        "poisson": m["poisson"],
        "groups": m["groups"],
        "plans": m["plans"],
        "rel_l2_vs_fp64": m["rel_l2_vs_fp64"],
        "e2e": {"value": total / t_srv / 1e9, "unit": "GB/s", "h2d_bytes_per_step": m["h2d_bytes"],
                "d2h_bytes_per_step": m["d2h_bytes"]},
        "clocks": m["clocks"],
    }
    print(json.dumps(line), flush=True)
    return 0


# --- CPU oracle beside the GPU workloads ---------------------------------------------


def oracle_seconds(shape, axes, sample_rows=None, seconds: float = 4.0):
    """Seconds the CPU oracle (reikna's algorithm restated, all host threads) takes
    for one complex64 transform of ``shape`` over ``axes``; with ``sample_rows`` it
    times that many rows of the first axis (not transformed) and scales up.
    Returns (seconds, threads, sample description)."""
    import numpy

    from oracle import oracle

    threads = os.cpu_count() or 1
    rows = shape[0]
    sub = tuple(shape) if not sample_rows or 0 in axes else (min(sample_rows, rows),) + tuple(shape[1:])
    rng = numpy.random.default_rng(3)
    x = (rng.standard_normal(sub) + 1j * rng.standard_normal(sub)).astype(numpy.complex64)
    plan = oracle.Plan(sub, axes)
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < 2 or (time.perf_counter() < t_end and len(times) < 20):
        t0 = time.perf_counter()
        plan(x, threads=threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times[1:]) if len(times) > 2 else times[-1]
    return t * rows / sub[0], threads, f"{list(sub)} over axes {list(axes)}" + (f", scaled to {rows} rows" if sub[0] != rows else "")


# --- batched launch -----------------------------------------------------------------


def measure_batch(dev, steps: int, warmup: int, modes=("calls", "graph", "graph_par", "persistent", "auto")):
    """Mixed-size batch: 1000 x 3001 (axis 1, Bluestein), 1000 x 1000 (both axes) and a
    1000 x 1000 float32 real-to-complex transform cropped to 1000 x 501, run as plain
    per-call execution and as one batch in each of ``modes``.  Returns (results by
    mode, algorithmic bytes per step)."""
    import numpy
    import torch

    from reikna_b200 import transformations as tr
    from reikna_b200.batch import BatchedFFT
    from reikna_b200.fft import FFT

    rng4, rng5, rng6 = (numpy.random.default_rng(s) for s in (4, 5, 6))
    xa = (rng4.standard_normal((1000, 3001)) + 1j * rng4.standard_normal((1000, 3001))).astype(numpy.complex64)
    xb = (rng5.standard_normal((1000, 1000)) + 1j * rng5.standard_normal((1000, 1000))).astype(numpy.complex64)
    xc = rng6.uniform(-1, 1, (1000, 1000)).astype(numpy.float32)
    ta, tb, tc = (torch.from_numpy(x).to(dev) for x in (xa, xb, xc))
    fa = FFT(ta, axes=(1,))
    fb = FFT(tb, axes=(0, 1))
    r2c = tr.real_to_complex(tc)
    fc = FFT(r2c.parameter.output)
    fc.parameter.input.connect(r2c, r2c.parameter.output, real_input=r2c.parameter.input)
    crop = tr.crop_frequencies(fc.parameter.output)
    fc.parameter.output.connect(crop, crop.parameter.input, half=crop.parameter.output)
    comps = [fa, fb, fc]
    outs = [torch.empty_like(ta), torch.empty_like(tb), torch.empty((1000, 501), dtype=torch.complex64, device=dev)]
    args_list = [(o, i) for o, i in zip(outs, (ta, tb, tc))]
    # B_alg per member: P_min (input + output bytes); M = 8192 (P 1), 2048^2 (P 2), 2048^2 (P 2)
    b_alg = 1 * (2 * 24_008_000) + 2 * (2 * 8_000_000) + 2 * (4_000_000 + 4_008_000)
    refs = [
        numpy.fft.fft(xa.astype(numpy.complex128), axis=1),
        numpy.fft.fft2(xb.astype(numpy.complex128)),
        numpy.fft.rfft2(xc.astype(numpy.float64)),
    ]

    def timed(fn, reps):
        for _ in range(max(3, warmup)):
            fn()
        torch.cuda.synchronize(dev)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(reps):
            fn()
        s1.record()
        torch.cuda.synchronize(dev)
        return s0.elapsed_time(s1) / reps

    reps = max(1, min(steps, 200))
    singles = [c.compile(dev) for c in comps]

    def plain():
        for cc, (o, i) in zip(singles, args_list):
            cc(None, o, i)

    res = {"plain_per_call": {"us": timed(plain, reps) * 1e3}}
    # each member alone: the batch cannot finish before its longest member, so
    # plain / max(member) bounds any batching speed-up
    alone = []
    for cc, (o, i) in zip(singles, args_list):
        alone.append(timed(lambda cc=cc, o=o, i=i: cc(None, o, i), reps) * 1e3)
    res["plain_per_call"]["members_alone_us"] = alone
    res["plain_per_call"]["max_speedup_bound"] = res["plain_per_call"]["us"] / max(alone)
    plain()
    torch.cuda.synchronize(dev)
    res["plain_per_call"]["rel_l2_vs_fp64"] = [
        float(numpy.linalg.norm((o.cpu().numpy() - r).ravel()) / numpy.linalg.norm(r.ravel())) for o, r in zip(outs, refs)]
    for mode in modes:
        bat = BatchedFFT(comps, device=dev, mode=mode)
        ms = timed(lambda: bat(None, args_list), reps)
        errs = [float(numpy.linalg.norm((o.cpu().numpy() - r).ravel()) / numpy.linalg.norm(r.ravel())) for o, r in zip(outs, refs)]
        entry = {"us": ms * 1e3, "rel_l2_vs_fp64": errs, "chosen": list(bat.chosen)}
        if mode == "persistent":
            entry["launch"] = bat._variant.batch.info()
        if mode == "auto":
            entry["tried"] = bat.tuning.get("tried") if bat.tuning else None
        res[mode] = entry
        bat.close()
    for k, v in res.items():
        v["gbs"] = b_alg / (v["us"] / 1e6) / 1e9
    return res, b_alg


def run_batch(args, rank: int, world: int, local_rank: int) -> int:
    """The mixed-size batch (``measure_batch``) in every batching mode, autotuned."""
    import torch

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    res, b_alg = measure_batch(dev, args.steps, args.warmup)
    reps = max(1, min(args.steps, 200))
    best = min((k for k in res if k != "plain_per_call"), key=lambda k: res[k]["us"])
    cpu_s, cpu_threads, samples = 0.0, 1, []
    if not args.no_cpu_baseline:
        # the real-input member runs on the CPU as the complex transform it reduces to
        for shape, axes, rows in (((1000, 3001), (1,), 100), ((1000, 1000), (0, 1), None), ((1000, 1000), (0, 1), None)):
            t, cpu_threads, desc = oracle_seconds(shape, axes, rows)
            cpu_s += t
            samples.append(desc)
    line = {
        "metric": METRIC,
        "value": res["auto"]["gbs"],
        "unit": "GB/s",
        "n_gpus": 1,
        "steps": reps,
        "warmup": args.warmup,
        "ms_per_step": res["auto"]["us"] / 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "batch_1000x3001_1000x1000_r2c1000x1000", "bytes_per_step_algorithmic": b_alg,
                   "fastest_mode": best},
        "modes": res,
        "speedup_vs_plain": res["plain_per_call"]["us"] / res["auto"]["us"],
    }
    if cpu_s:
        line["cpu_baseline"] = {"value": b_alg / cpu_s / 1e9, "unit": "GB/s", "cores": cpu_threads, "kind": "port",
                                "sample": "; ".join(samples), "ms_per_step": cpu_s * 1e3}
    print(json.dumps(line), flush=True)
    return 0


# --- precision mode ---------------------------------------------------------------


def measure_precision(dev, steps: int, warmup: int):
    """16384 x 1024 complex64 along the last axis, plain FP32 against the tensor-core
    split-precision mode, on N(0,1) data and on a 60 dB variant (components
    +-10^U(-3,0)).  Returns (results, algorithmic bytes per step)."""
    import numpy
    import torch

    from reikna_b200 import _native as N
    from reikna_b200.fft import FFT

    shape = (16384, 1024)
    nbytes = shape[0] * shape[1] * 8
    b_alg = 2 * nbytes  # P_min = 1
    peak, peak_kind = peaks()
    out = {}
    for label, seed in (("normal", 7), ("sixty_db", 8)):
        rng = numpy.random.default_rng(seed)
        if label == "normal":
            x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(numpy.complex64)
        else:
            mag = 10 ** rng.uniform(-3, 0, (2,) + shape)
            sgn = rng.choice([-1.0, 1.0], (2,) + shape)
            x = (sgn[0] * mag[0] + 1j * sgn[1] * mag[1]).astype(numpy.complex64)
        ref = numpy.fft.fft(x.astype(numpy.complex128), axis=1)
        xs = [torch.from_numpy(x).to(dev), torch.from_numpy(x).to(dev)]
        ys = [torch.empty_like(xs[0]) for _ in range(2)]
        res = {}
        for mode, flags in (("fp32", 0), ("split_tc", N.FLAG_SPLIT_TC)):
            comp = FFT(xs[0], axes=(1,)).compile(dev, flags=flags)
            plan = comp._runner.plan
            for k in range(max(3, warmup)):
                comp(None, ys[k % 2], xs[k % 2])
            torch.cuda.synchronize(dev)
            nsteps = max(1, min(steps, 500))
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record()
            for k in range(nsteps):
                comp(None, ys[k % 2], xs[k % 2])
            s1.record()
            torch.cuda.synchronize(dev)
            ms = s0.elapsed_time(s1) / nsteps
            comp(None, ys[0], xs[0])
            y = ys[0].cpu().numpy()
            err = float(numpy.linalg.norm((y - ref).ravel()) / numpy.linalg.norm(ref.ravel()))
            res[mode] = {
                "gbs": b_alg / (ms / 1e3) / 1e9,
                "hbm_frac": b_alg / (ms / 1e3) / 1e9 / peak,
                "us_per_step": ms * 1e3,
                "rel_l2_vs_fp64": err,
                "tensor_core_passes": plan.tc_passes,
                "kernel": plan.describe()["passes"][0]["note"],
            }
        out[label] = res
    return out, b_alg


def run_precision(args, rank: int, world: int, local_rank: int) -> int:
    """FP32 against the tensor-core split mode (``measure_precision``)."""
    import torch

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    shape = (16384, 1024)
    peak, peak_kind = peaks()
    out, b_alg = measure_precision(dev, args.steps, args.warmup)
    cpu = None
    if not args.no_cpu_baseline:
        t, threads, desc = oracle_seconds(shape, (1,), 1024)
        cpu = {"value": b_alg / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "port", "sample": desc,
               "ms_per_step": t * 1e3}
    line = {
        "metric": METRIC,
        "value": out["normal"]["split_tc"]["gbs"],
        "unit": "GB/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": out["normal"]["split_tc"]["us_per_step"] / 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "tf32x2-split/f32-acc",
        "data": "synthetic",
        "config": {"workload": "precision_16384x1024_complex64", "shape": list(shape), "axes": [1],
                   "bytes_per_step_algorithmic": b_alg, "l2": "inputs larger than L2, two buffer sets alternate",
                   "peak_gbs": peak, "peak_kind": peak_kind},
        "results": out,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# --- next rows: spectrogram, FFTShift, Transpose, real transforms ------------------


def run_next(args, rank: int, world: int, local_rank: int) -> int:
    """The computations around the FFT at their workload sizes, each through its public
    computation API: the spectrogram of a 2^22-sample float32 signal (Hann 1024, hop
    256; frame-major and transposed), FFTShift and Transpose of 4096 x 4096 complex64,
    and the half-length real transforms of 16384 rows of 1024 float32 samples (RFFT,
    IRFFT, APRFFT, IAPRFFT).  Two buffer sets alternate (each op moves more than the
    126 MB L2 in total per pair of steps, and the big ones more than L2 per step);
    device time from CUDA events over the timed steps."""
    import numpy
    import torch

    from reikna_b200.algorithms import Transpose
    from reikna_b200.fft import APRFFT, FFTShift, IAPRFFT, IRFFT, RFFT
    from reikna_b200.spectrogram import frames, spectrogram

    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    peak, peak_kind = peaks()
    rng = numpy.random.default_rng(9)
    steps = max(1, min(args.steps, 500))

    def timed(call, pairs):
        for k in range(max(3, args.warmup)):
            call(*pairs[k % 2])
        torch.cuda.synchronize(dev)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for k in range(steps):
            call(*pairs[k % 2])
        s1.record()
        torch.cuda.synchronize(dev)
        return s0.elapsed_time(s1) / steps

    def entry(us, b_alg, err, launches):
        gbs = b_alg / (us / 1e6) / 1e9
        return {"us": us, "gbs": gbs, "hbm_frac": gbs / peak, "bytes_algorithmic": b_alg,
                "rel_l2_vs_fp64": err, "launches": launches}

    def rel(a, b):
        a = numpy.asarray(a, numpy.complex128)
        b = numpy.asarray(b, numpy.complex128)
        return float(numpy.linalg.norm((a - b).ravel()) / numpy.linalg.norm(b.ravel()))

    res = {}
    # spectrogram: 2^22 samples, N(0,1) plus 8 sinusoids
    n_sig, nfft, hop = 2**22, 1024, 256
    t_idx = numpy.arange(n_sig)
    sig = rng.standard_normal(n_sig)
    for _ in range(8):
        sig += rng.uniform(0.1, 2) * numpy.sin(2 * numpy.pi * rng.uniform(0, 0.5) * t_idx + rng.uniform(0, 2 * numpy.pi))
    sig = sig.astype(numpy.float32)
    nfr = frames(n_sig, nfft, hop)
    idx = numpy.arange(nfr)[:, None] * hop + numpy.arange(nfft)[None, :]
    win = 0.5 * (1 - numpy.cos(2 * numpy.pi * numpy.arange(nfft) / (nfft - 1)))
    spec_ref = numpy.abs(numpy.fft.rfft(sig.astype(numpy.float64)[idx] * win, axis=1))
    sigs = [torch.from_numpy(sig).to(dev) for _ in range(2)]
    for label, transposed in (("spectrogram", False), ("spectrogram_transposed", True)):
        cc = spectrogram(n_sig, nfft, hop, transposed=transposed).compile(dev)
        shape = (nfft // 2 + 1, nfr) if transposed else (nfr, nfft // 2 + 1)
        outs = [torch.empty(shape, dtype=torch.float32, device=dev) for _ in range(2)]
        us = timed(lambda o, i: cc(None, o, i), list(zip(outs, sigs))) * 1e3
        got = outs[0].cpu().numpy()
        res[label] = entry(us, n_sig * 4 + nfr * (nfft // 2 + 1) * 4, rel(got.T if transposed else got, spec_ref),
                           cc.launches)
    del spec_ref, idx
    # FFTShift and Transpose of 4096 x 4096 complex64 (134 MB each way)
    x = (rng.standard_normal((4096, 4096)) + 1j * rng.standard_normal((4096, 4096))).astype(numpy.complex64)
    xs = [torch.from_numpy(x).to(dev) for _ in range(2)]
    ys = [torch.empty_like(xs[0]) for _ in range(2)]
    cc = FFTShift(xs[0]).compile(dev)
    us = timed(lambda o, i: cc(None, o, i), list(zip(ys, xs))) * 1e3
    res["fftshift_4096x4096"] = entry(us, 2 * x.nbytes, rel(ys[0].cpu().numpy(), numpy.fft.fftshift(x)), cc.launches)
    cc = Transpose(xs[0]).compile(dev)
    us = timed(lambda o, i: cc(None, o, i), list(zip(ys, xs))) * 1e3
    res["transpose_4096x4096"] = entry(us, 2 * x.nbytes, rel(ys[0].cpu().numpy(), x.T), cc.launches)
    del x, xs, ys
    # real transforms: 16384 x 1024 float32
    shape = (16384, 1024)
    xr = rng.uniform(-1, 1, shape).astype(numpy.float32)
    full = numpy.fft.rfft(xr.astype(numpy.float64), axis=1)
    harm = numpy.fft.rfft(numpy.concatenate([xr, -xr], axis=1).astype(numpy.float64), axis=1)[:, 1::2]
    xrs = [torch.from_numpy(xr).to(dev) for _ in range(2)]
    specs = [torch.empty((16384, 513), dtype=torch.complex64, device=dev) for _ in range(2)]
    hs = [torch.empty((16384, 512), dtype=torch.complex64, device=dev) for _ in range(2)]
    backs = [torch.empty_like(xrs[0]) for _ in range(2)]
    for label, comp, outs, ins, ref, b_alg in (
        ("rfft_16384x1024", RFFT(xrs[0]), specs, xrs, full, xr.nbytes + 16384 * 513 * 8),
        ("irfft_16384x1024", IRFFT(specs[0]), backs, specs, xr, xr.nbytes + 16384 * 513 * 8),
        ("aprfft_16384x1024", APRFFT(xrs[0]), hs, xrs, harm, xr.nbytes + 16384 * 512 * 8),
        ("iaprfft_16384x1024", IAPRFFT(hs[0]), backs, hs, xr, xr.nbytes + 16384 * 512 * 8),
    ):
        cc = comp.compile(dev)
        us = timed(lambda o, i: cc(None, o, i), list(zip(outs, ins))) * 1e3
        res[label] = entry(us, b_alg, rel(outs[0].cpu().numpy(), ref), cc.launches)
    cpu = None
    if not args.no_cpu_baseline:
        # the oracle's FFT of the windowed frames (reikna's composition on the CPU),
        # a bounded sample of frames scaled to the whole signal
        from oracle import oracle

        sample = 2048
        fr = (sig[numpy.arange(sample)[:, None] * hop + numpy.arange(nfft)[None, :]] * win.astype(numpy.float32)).astype(
            numpy.complex64)
        plan = oracle.Plan(fr.shape, (1,))
        times = []
        t_end = time.perf_counter() + 6.0
        while len(times) < 3 or (time.perf_counter() < t_end and len(times) < 30):
            t0 = time.perf_counter()
            numpy.abs(plan(fr, threads=os.cpu_count())[:, : nfft // 2 + 1])
            times.append(time.perf_counter() - t0)
        t = statistics.median(times[1:]) * nfr / sample
        cpu = {"value": res["spectrogram"]["bytes_algorithmic"] / t / 1e9, "unit": "GB/s", "cores": os.cpu_count(),
               "kind": "port", "sample": f"{sample} of {nfr} frames (window, complex64 FFT, magnitude, crop), scaled",
               "ms_per_step": t * 1e3}
    head = res["spectrogram_transposed"]
    line = {
        "metric": METRIC,
        "value": head["gbs"],
        "unit": "GB/s",
        "n_gpus": 1,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": head["us"] / 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "next_rows_spectrogram_2^22_fftshift_transpose_4096^2_real_16384x1024",
                   "l2": "two buffer sets alternate", "peak_gbs": peak, "peak_kind": peak_kind},
        "results": res,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["own", "reference"], default="own")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="fft3d: skip the compact C1/C2b/C3/C4/C5 measurements after the headline")
    ap.add_argument("--serve-sample", type=int, default=300,
                    help="fft3d: requests of the serving stream measured in the configs object")
    ap.add_argument("--workload", choices=["fft3d", "serve", "precision", "batch", "next"], default="fft3d",
                    help="fft3d: the headline 256^3 transform; serve: the request stream; "
                    "precision: FP32 against the tensor-core split mode on 16384 x 1024; "
                    "batch: the mixed-size batch in every batching mode; next: spectrogram, FFTShift, "
                    "Transpose and the real transforms")
    ap.add_argument("--requests", type=int, default=1000, help="serve: requests in the stream")
    ap.add_argument("--streams", type=int, default=4, help="serve: compute streams of the server")
    ap.add_argument("--load", type=float, default=0.7, help="serve: Poisson rate / served burst rate")
    ap.add_argument("--serve-data", choices=["host", "device"], default="host",
                    help="serve: request data in pinned host memory or already in device memory")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "serve":
        return run_serve(args, rank, world, local_rank)
    if args.workload == "precision":
        return run_precision(args, rank, world, local_rank)
    if args.workload == "batch":
        return run_batch(args, rank, world, local_rank)
    if args.workload == "next":
        return run_next(args, rank, world, local_rank)
    return run_own(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
