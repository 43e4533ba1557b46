"""Batched execution of several compiled FFT computations.

The reference runs every compiled computation as its own chain of kernel launches
(``ComputationCallable.__call__``, reikna/core/computation.py:766).  A
:class:`BatchedFFT` runs a fixed list of computations (any shapes, axes and
connected transformations) as one unit, in one of three modes:

``"calls"``
    one ``rk_fft_execute`` per member, back to back on the stream (the plain path);
``"graph"``
    the same launches captured once into a CUDA graph and replayed (one graph launch
    per call; recaptured when the argument pointers change);
``"graph_par"``
    as ``"graph"``, with every member on its own branch of the graph (forked from
    and joined back to the calling stream), so the kernels of independent members
    run concurrently and a member that leaves SMs idle (a one-CTA-an-SM Bluestein
    pass, a short final wave) shares them with the others;
``"persistent"``
    ``rk_batch_execute``: one persistent kernel whose CTAs pull the tiles of every
    member's passes from a dependency-ordered task list, so small members fill the
    GPU together and a member's next pass starts as soon as its previous pass is done.

``mode="auto"`` times every applicable (mode, plan flags) candidate on the first
call's arguments, keeps the fastest, and remembers the choice in a JSON cache keyed by
the members' native descriptors (``RK_AUTOTUNE_CACHE``, default
``~/.cache/reikna_b200/autotune.json``).
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

from . import _native as N

MODES = ("calls", "graph", "graph_par", "persistent")

# bumped when the candidate set changes, so that older cached choices are re-tuned
_TUNE_VERSION = b"3"


def _cache_path() -> Path:
    p = os.environ.get("RK_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "reikna_b200" / "autotune.json"


def _desc_key(descs) -> str:
    h = hashlib.sha256(_TUNE_VERSION)
    for d in descs:
        h.update(bytes(d))
    return h.hexdigest()[:32]


def _load_cache() -> dict:
    try:
        return json.loads(_cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store_cache(key: str, entry: dict) -> None:
    path = _cache_path()
    try:
        cache = _load_cache()
        cache[key] = entry
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass  # a read-only home only loses the cache


class _Variant:
    """The members compiled with one set of plan flags, runnable in one mode."""

    def __init__(self, comps, device, mode: str, flags: int):
        self.mode = mode
        self.flags = flags
        self.device = device
        self.callables = [c.compile(device, flags=flags) for c in comps]
        self.plans = [c._runner.plan for c in self.callables]
        self.batch = N.Batch(self.plans) if mode == "persistent" else None
        self._graphs = {}
        self._branches = None

    def bind(self, args_list):
        calls = []
        for cc, args in zip(self.callables, args_list):
            if isinstance(args, dict):
                bound = cc.signature.bind_with_defaults((), args, cast=True)
            else:
                bound = cc.signature.bind_with_defaults(tuple(args), {}, cast=True)
            calls.append(cc._runner.bind(bound.arguments))
        return calls

    def _launch_calls(self, calls, stream: int) -> None:
        if self.mode == "graph_par":
            self._launch_branches(calls)
            return
        for plan, (outs, ins, inverse, scalars) in zip(self.plans, calls):
            plan.execute(outs, ins, inverse=inverse, scalars=scalars, stream=stream)

    def _launch_branches(self, calls) -> None:
        """Each member on its own stream, forked from and joined back to the current
        torch stream (the capture stream while a graph is captured).  Members are
        distinct plans with their own temporaries, so they may run at once."""
        import torch

        if self._branches is None:
            self._branches = [torch.cuda.Stream(device=self.device) for _ in self.plans]
        main = torch.cuda.current_stream(self.device)
        for s, plan, (outs, ins, inverse, scalars) in zip(self._branches, self.plans, calls):
            s.wait_stream(main)
            plan.execute(outs, ins, inverse=inverse, scalars=scalars, stream=s.cuda_stream)
        for s in self._branches:
            main.wait_stream(s)

    def run(self, calls, stream: int) -> None:
        if self.mode == "persistent":
            self.batch.execute(calls, stream=stream)
        elif self.mode == "calls":
            self._launch_calls(calls, stream)
        else:
            self._replay(calls, stream)

    def _replay(self, calls, stream: int) -> None:
        import torch

        key = tuple((tuple(o), tuple(i), inv, tuple(complex(s) for s in sc)) for o, i, inv, sc in calls)
        ext = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
        g = self._graphs.get(key)
        if g is None:
            if len(self._graphs) >= 8:
                self._graphs.clear()
            side = torch.cuda.Stream()
            # the eager run and the capture come after the caller's pending work on
            # its stream (which may still be writing the inputs or reading the outputs)
            side.wait_stream(ext)
            # one eager run first: per-call host state (tensor maps, staging) is settled
            # before capture
            with torch.cuda.stream(side):
                self._launch_calls(calls, side.cuda_stream)
            side.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                self._launch_calls(calls, side.cuda_stream)
            self._graphs[key] = g
        with torch.cuda.stream(ext):
            g.replay()

    def close(self) -> None:
        self._graphs.clear()
        if self.batch is not None:
            self.batch.close()
            self.batch = None


class BatchedFFT:
    """Run a fixed list of computations as one batch.

    :param computations: ``reikna_b200`` computations (e.g. ``FFT`` objects with
        transformations connected), not yet compiled.
    :param device: torch device (default: the current CUDA device).
    :param mode: ``"calls"``, ``"graph"``, ``"graph_par"``, ``"persistent"`` or ``"auto"``.
    :param flags: plan flags for a fixed mode (``"persistent"`` adds
        ``FLAG_BATCHABLE``: only passes with a batched tile body).

    Call as ``batched(stream, [args_0, args_1, ...])`` where ``args_i`` is the
    positional tuple (or keyword dict) member i's compiled callable takes.
    Asynchronous on ``stream``, like a single computation call.
    """

    def __init__(self, computations, device=None, mode: str = "auto", flags: int = 0):
        import torch

        if mode not in MODES + ("auto",):
            raise ValueError(f"unknown batch mode {mode!r}")
        self.computations = list(computations)
        if not self.computations:
            raise ValueError("a batch needs at least one computation")
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device) if not isinstance(device, torch.device) else device
        self.mode = mode
        self._flags = flags
        self._variant = None
        self.tuning = None
        if mode != "auto":
            f = flags | (N.FLAG_BATCHABLE if mode == "persistent" else 0)
            self._variant = _Variant(self.computations, self.device, mode, f)

    def key(self) -> str:
        return _desc_key([c.native_descriptor(0)[0] for c in self.computations])

    def candidates(self):
        """(mode, flags) pairs the autotuner tries: the launch mode crossed with the
        members' kernel-shape choices (``reikna_b200.autotune.candidates``: TMA
        staging, plane tile shape, Bluestein radix plan / fusion)."""
        from .autotune import candidates as member_flags

        shapes = [0, N.FLAG_NO_TMA]
        for c in self.computations:
            try:
                for f in member_flags(c):
                    if f not in shapes and f != N.FLAG_SPLIT_TC:
                        shapes.append(f)
            except (N.NativeError, NotImplementedError, ValueError, AttributeError):
                pass
        out = [("calls", 0), ("calls", N.FLAG_NO_TMA)]
        out += [("graph", f) for f in shapes]
        if len(self.computations) > 1:
            out += [("graph_par", f) for f in shapes]
        out.append(("persistent", N.FLAG_BATCHABLE))
        return out

    @property
    def chosen(self):
        v = self._variant
        return None if v is None else (v.mode, v.flags)

    def _tune(self, args_list, stream: int) -> None:
        import torch

        key = self.key()
        cached = _load_cache().get(key)
        if cached is not None:
            try:
                self._variant = _Variant(self.computations, self.device, cached["mode"], int(cached["flags"]))
                self.tuning = {"cached": True, **cached}
                return
            except (N.NativeError, NotImplementedError, ValueError):
                pass
        results = []
        best = None
        ext = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
        for mode, flags in self.candidates():
            try:
                v = _Variant(self.computations, self.device, mode, flags)
                calls = v.bind(args_list)
            except (N.NativeError, NotImplementedError, ValueError):
                continue  # e.g. a member with no batched variant
            with torch.cuda.stream(ext):
                for _ in range(3):
                    v.run(calls, stream)
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                reps = 10
                s.record()
                for _ in range(reps):
                    v.run(calls, stream)
                e.record()
            e.synchronize()
            ms = s.elapsed_time(e) / reps
            results.append({"mode": mode, "flags": flags, "ms": ms})
            if best is None or ms < best[0]:
                if best is not None:
                    best[1].close()
                best = (ms, v)
            else:
                v.close()
        if best is None:
            raise N.NativeError("no batch mode could run these computations")
        self._variant = best[1]
        entry = {"mode": best[1].mode, "flags": best[1].flags, "ms": best[0], "tried": results}
        self.tuning = {"cached": False, **entry}
        _store_cache(key, entry)

    def __call__(self, stream, args_list) -> None:
        from .core.computation import stream_handle

        h = stream_handle(stream)
        if len(args_list) != len(self.computations):
            raise ValueError(f"expected {len(self.computations)} argument sets, got {len(args_list)}")
        if self._variant is None:
            self._tune(args_list, h)
        v = self._variant
        v.run(v.bind(args_list), h)

    def close(self) -> None:
        if self._variant is not None:
            self._variant.close()
