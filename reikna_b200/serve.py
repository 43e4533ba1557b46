"""Serving loop: continuous batching of FFT and spectrogram requests on one GPU.

The reference has no serving layer; its callers run one compiled computation per
array shape and wait for it (``ComputationCallable.__call__``,
reikna/core/computation.py:766).  :class:`FFTServer` takes requests with host data as
they arrive and keeps the GPU busy with them:

* **Classes and coalescing.**  Requests of the same class (1-D transforms of the same
  length and direction, 2-D transforms of the same shape, spectrograms of the same
  signal length) that are waiting together are stacked into one device buffer and
  transformed by a few calls of resident plans: a group of ``B`` rows runs as one plan
  call per set bit of ``B`` (plans of 2^k rows), so a handful of plans per class
  serves every batch size without padding work.
* **Continuous admission.**  A group is launched whenever a stream slot and device
  memory are free; requests that arrive while others are on the GPU join the next
  group of their class.  Device memory in flight (staging buffers plus resident plans)
  stays under ``memory_budget`` bytes.
* **Overlap.**  A group is a three-stage pipeline: uploads on one stream, transforms
  on a compute stream, downloads on a third, chained by events, so uploads of later
  groups run while earlier ones compute and download.  Each class is bound to one of
  ``streams`` compute streams (assigned round-robin as classes first appear), up to
  ``depth`` groups in flight a stream.  A class's plans are only ever used from its
  own stream, in order, which is what a plan's temporaries need (they serve one call
  at a time).
* **Resident plans.**  Plans stay compiled in a cache of at most ``plan_budget``
  device bytes (least recently used out); :meth:`FFTServer.prepare` compiles every
  plan size a set of classes can need ahead of the traffic.
* **Accounting.**  Every request records arrival, launch and completion times; the
  caller reads latencies off the finished requests.

Inputs are host tensors (pinned ones make the copies asynchronous); results come back
in pinned host tensors the server allocates.  In-place transforms keep one staging
buffer per group.  Device tensors are accepted too: the server orders its work after
the submitter's stream as it was at :meth:`FFTServer.submit` (an event recorded there)
and keeps the tensors alive for its own streams (``record_stream``); a consumer of a
device result waits on the request's ``event``.

**Failures** stay with the requests they belong to.  A request whose staging alone
exceeds ``memory_budget`` is rejected at submission (``status == "rejected"``); a
waiting request can be cancelled (:meth:`FFTServer.cancel`); a group whose plan cannot
be compiled, or whose buffers cannot be allocated, or whose launch raises, ends with
``status == "failed"`` and the exception in ``error``, while every other group carries
on.  ``done`` is set for every final status.
"""

from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy

from .fft import FFT
from .spectrogram import frames as _frames
from .spectrogram import spectrogram as _spectrogram


def binary_pieces(n: int) -> list[int]:
    """Powers of two, largest first, that sum to ``n`` (one plan call each)."""
    if n < 1:
        raise ValueError("a group has at least one row")
    out, bit = [], 1 << (n.bit_length() - 1)
    while bit:
        if n & bit:
            out.append(bit)
        bit >>= 1
    return out


@dataclass(eq=False)
class FFTRequest:
    """One request.

    ``kind``: ``"fft1d"`` (``data``: complex64 (rows, n), transformed along the last
    axis), ``"fft2d"`` (complex64 (n1, n2), both axes) or ``"spectrogram"`` (float32
    (length,), ``nfft``/``hop`` frames, magnitudes of the first ``nfft // 2 + 1`` bins).
    """

    kind: str
    data: object
    inverse: int = 0
    nfft: int = 1024
    hop: int = 256
    out: object = None      # optional host tensor that receives the result
    result: object = None
    arrival: float = 0.0
    launched: float = 0.0
    finished: float = 0.0
    done: bool = False
    status: str = "new"     # waiting, running, done, failed, cancelled, rejected
    error: object = None    # the exception of a failed or rejected request
    ready: object = None    # event on the submitter's stream (device inputs / outputs)
    event: object = None    # completion event of the request's group on the GPU

    def key(self):
        shape = tuple(self.data.shape)
        if self.kind == "fft1d":
            if len(shape) != 2:
                raise ValueError("fft1d requests are (rows, n) arrays")
            return ("fft1d", shape[1], int(self.inverse))
        if self.kind == "fft2d":
            if len(shape) != 2:
                raise ValueError("fft2d requests are (n1, n2) arrays")
            return ("fft2d", shape[0], shape[1], int(self.inverse))
        if self.kind == "spectrogram":
            if len(shape) != 1:
                raise ValueError("spectrogram requests are 1-D signals")
            return ("spectrogram", shape[0], int(self.nfft), int(self.hop))
        raise ValueError(f"unknown request kind {self.kind!r}")

    def rows(self) -> int:
        return int(self.data.shape[0]) if self.kind == "fft1d" else 1

    def in_bytes(self) -> int:
        return int(numpy.prod(self.data.shape)) * self.data.element_size()

    def out_shape(self):
        if self.kind == "spectrogram":
            return (_frames(self.data.shape[0], self.nfft, self.hop), self.nfft // 2 + 1)
        return tuple(self.data.shape)

    def on_device(self) -> bool:
        return bool(getattr(self.data, "is_cuda", False) or getattr(self.out, "is_cuda", False))

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class AdmissionError(MemoryError):
    """A request needs more staging memory than the server's whole budget."""


def _computation(key, rows: int):
    """The computation that serves ``rows`` stacked requests of class ``key``."""
    import torch

    from .core import ArrayMetadata

    kind = key[0]
    if kind == "fft1d":
        return FFT(ArrayMetadata((rows, key[1]), numpy.complex64), axes=(1,))
    if kind == "fft2d":
        return FFT(ArrayMetadata((rows, key[1], key[2]), numpy.complex64), axes=(1, 2))
    del torch
    return _spectrogram(key[1], key[2], key[3])


class PlanCache:
    """Compiled computations by (class, rows), least recently used out beyond
    ``budget`` device bytes (freeing a plan's memory waits for the device)."""

    def __init__(self, device, budget: int):
        self.device = device
        self.budget = int(budget)
        self._plans = collections.OrderedDict()
        self.bytes = 0
        self.compiles = 0
        self.evictions = 0
        self.compile_s = 0.0

    def get(self, key, rows: int):
        k = (key, rows)
        cc = self._plans.get(k)
        if cc is None:
            t0 = time.perf_counter()
            cc = _computation(key, rows).compile(self.device)
            self.compile_s += time.perf_counter() - t0
            self.compiles += 1
            self.bytes += cc._runner.plan.device_bytes
            self._plans[k] = cc
            while self.bytes > self.budget and len(self._plans) > 1:
                self._evict_oldest()
        else:
            self._plans.move_to_end(k)
        return cc

    def _evict_oldest(self) -> None:
        _, cc = self._plans.popitem(last=False)
        self.bytes -= cc._runner.plan.device_bytes
        cc._runner.plan.close()
        self.evictions += 1


@dataclass(eq=False)
class _Group:
    key: tuple
    requests: list
    stream_index: int
    bytes: int
    event: object = None
    buffers: list = field(default_factory=list)
    error: object = None


class FFTServer:
    """Continuous-batching FFT server on one GPU (see the module docstring).

    :param device: torch CUDA device (default: current).
    :param memory_budget: device bytes of request data in flight (admission budget).
    :param streams: CUDA streams the classes are spread over.
    :param depth: groups in flight per stream.
    :param max_group_bytes: input bytes above which a group takes no more requests.
    :param plan_budget: device bytes of resident plans (temporaries and tables).
    """

    def __init__(self, device=None, memory_budget: int = 40 << 30, streams: int = 4, depth: int = 2,
                 max_group_bytes: int = 256 << 20, plan_budget: int = 40 << 30):
        import torch

        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        self.memory_budget = int(memory_budget)
        self.depth = int(depth)
        self.max_group_bytes = int(max_group_bytes)
        self.nstreams = int(streams)
        self.streams = None          # created with the first launch
        self.upload = self.download = None
        self.plans = PlanCache(self.device, plan_budget)
        self._class_stream = {}
        self._waiting = collections.OrderedDict()  # class key -> deque of requests
        self._inflight = [collections.deque() for _ in range(streams)]
        self._staged = 0
        self.groups = 0
        self.completed = 0
        self.failed = 0
        self.rejected = 0
        self.cancelled = 0

    def _streams(self):
        import torch

        if self.streams is None:
            with torch.cuda.device(self.device):
                self.streams = [torch.cuda.Stream(self.device) for _ in range(self.nstreams)]
                self.upload = torch.cuda.Stream(self.device)
                self.download = torch.cuda.Stream(self.device)
        return self.streams

    # -- intake ------------------------------------------------------------------
    def submit(self, req: FFTRequest, now: float | None = None) -> FFTRequest:
        """Queue ``req``.  A request whose staging alone is larger than the whole
        memory budget can never be admitted: it comes back with ``status ==
        "rejected"`` and an :class:`AdmissionError`.  For device inputs or outputs an
        event is recorded on the submitter's current stream; the server's work on the
        request waits for it."""
        key = req.key()
        req.arrival = time.perf_counter() if now is None else now
        if not self._direct([req]) and self.group_bytes([req]) > self.memory_budget:
            req.status, req.done, req.finished = "rejected", True, req.arrival
            req.error = AdmissionError(
                f"request stages {self.group_bytes([req])} bytes, over the {self.memory_budget}-byte budget")
            self.rejected += 1
            return req
        if req.on_device():
            import torch

            req.ready = torch.cuda.Event()
            req.ready.record(torch.cuda.current_stream(self.device))
        req.status = "waiting"
        self._waiting.setdefault(key, collections.deque()).append(req)
        return req

    def cancel(self, req: FFTRequest) -> bool:
        """Withdraw a request that is still waiting; True if it was.  A request already
        on the GPU runs to the end (its group shares buffers and launches)."""
        if req.status != "waiting":
            return False
        q = self._waiting.get(req.key())
        if q is None or req not in q:
            return False
        q.remove(req)
        req.status, req.done, req.finished = "cancelled", True, time.perf_counter()
        self.cancelled += 1
        return True

    @property
    def pending(self) -> int:
        return sum(len(q) for q in self._waiting.values()) + sum(
            len(g.requests) for d in self._inflight for g in d
        )

    # -- scheduling ----------------------------------------------------------------
    def stream_of(self, key) -> int:
        s = self._class_stream.get(key)
        if s is None:
            s = self._class_stream[key] = len(self._class_stream) % self.nstreams
        return s

    def _next_class(self):
        """The class with the oldest waiting request among those whose stream has a
        free slot."""
        best, t = None, None
        for key, q in self._waiting.items():
            if q and (t is None or q[0].arrival < t) and len(self._inflight[self.stream_of(key)]) < self.depth:
                best, t = key, q[0].arrival
        return best

    def prepare(self, requests) -> None:
        """Compile, ahead of traffic, every plan the classes of ``requests`` can use:
        one per power of two up to the most rows a group of the class can stack."""
        for r in requests:
            key = r.key()
            self.stream_of(key)
            if r.kind == "spectrogram":
                self.plans.get(key, 1)
                continue
            per_row = r.in_bytes() // r.rows()
            most = max(r.rows(), self.max_group_bytes // per_row)
            k = 1
            while k <= most:
                self.plans.get(key, k)
                k *= 2

    @staticmethod
    def group_bytes(reqs) -> int:
        """Device bytes a group stages: the stacked input plus a separate output
        when the result has another type or shape (spectrograms)."""
        b = sum(r.in_bytes() for r in reqs)
        for r in reqs:
            if r.kind == "spectrogram":
                b += int(numpy.prod(r.out_shape())) * 4
        return b

    @staticmethod
    def _direct(reqs) -> bool:
        """Device inputs with device outputs: transformed in place of staging."""
        return all(getattr(r.data, "is_cuda", False) and getattr(r.out, "is_cuda", False) for r in reqs)

    def _take(self, key):
        q = self._waiting[key]
        take = [q.popleft()]
        size = take[0].in_bytes()
        while q and size + q[0].in_bytes() <= self.max_group_bytes:
            size += q[0].in_bytes()
            take.append(q.popleft())
        return take

    def step(self) -> int:
        """Retire finished groups, then launch groups while streams and memory allow.
        Returns the number of groups launched (failed ones included)."""
        self._retire()
        launched = 0
        while True:
            key = self._next_class()
            if key is None:
                break
            s = self.stream_of(key)
            reqs = self._take(key)
            need = 0 if self._direct(reqs) else self.group_bytes(reqs)
            if self._staged and self._staged + need > self.memory_budget:
                # wait for memory: put the requests back at the head of their queue
                self._waiting[key].extendleft(reversed(reqs))
                break
            self._launch(key, reqs, s, need)
            launched += 1
        return launched

    # allocation of staging buffers (a separate method so that it can be replaced)
    def _alloc(self, shape, dtype):
        import torch

        return torch.empty(shape, dtype=dtype, device=self.device)

    def _plans_for(self, key, reqs):
        """Every compiled plan the group needs, before any of its work is queued, so
        that a compile or allocation failure leaves nothing in flight."""
        if key[0] == "spectrogram" or self._direct(reqs) and key[0] == "fft2d":
            return {1: self.plans.get(key, 1)}
        sizes = set()
        if self._direct(reqs):
            for r in reqs:
                sizes.update(binary_pieces(r.rows()))
        else:
            sizes.update(binary_pieces(sum(r.rows() for r in reqs)))
        return {k: self.plans.get(key, k) for k in sorted(sizes)}

    def _fail(self, reqs, err) -> None:
        now = time.perf_counter()
        for r in reqs:
            r.status, r.error, r.done, r.finished = "failed", err, True, now
        self.failed += len(reqs)

    def _launch(self, key, reqs, s: int, need: int) -> None:
        """Three-stage pipeline of one group: host-to-device copies on the upload
        stream, the transforms on the class's compute stream, device-to-host copies on
        the download stream, chained by events.  Uploads of later groups run while
        earlier groups compute and download (the link carries both directions at once).
        A failure before anything is queued fails the group's requests only; one after
        (a launch that raises) also waits for the group's queued work before its
        buffers are released."""
        import torch

        try:
            plans = self._plans_for(key, reqs)
        except Exception as e:  # noqa: BLE001 - a failure stays with its group
            self._fail(reqs, e)
            return
        streams = self._streams()
        stream = streams[s]
        now = time.perf_counter()
        g = _Group(key, reqs, s, need)
        for r in reqs:
            r.launched, r.status = now, "running"
        try:
            with torch.cuda.device(self.device):
                if self._direct(reqs):
                    g.bytes = 0
                    self._run_direct(key, reqs, plans, stream, g)
                else:
                    self._run_staged(key, reqs, plans, stream, g)
        except Exception as e:  # noqa: BLE001
            g.error = e
            with torch.cuda.device(self.device):
                # whatever was queued finishes before the buffers can go
                for st in (self.upload, stream):
                    ev = torch.cuda.Event()
                    ev.record(st)
                    self.download.wait_event(ev)
                g.event = torch.cuda.Event()
                g.event.record(self.download)
        for r in reqs:
            r.event = g.event
        self._staged += g.bytes
        self._inflight[s].append(g)
        self.groups += 1

    def _run_direct(self, key, reqs, plans, stream, g) -> None:
        """Device-resident requests with device outputs: no staging, each request is
        transformed from its input straight into its output on the class's stream,
        after the submitter's stream reached the point of submission."""
        import torch

        for r in reqs:
            if r.ready is not None:
                stream.wait_event(r.ready)
            r.data.record_stream(stream)
            r.out.record_stream(stream)
            if key[0] == "spectrogram":
                plans[1](stream, r.out, r.data)
            elif key[0] == "fft2d":
                plans[1](stream, r.out[None], r.data[None], key[-1])
            else:
                off = 0
                for piece in binary_pieces(r.rows()):
                    plans[piece](stream, r.out[off : off + piece], r.data[off : off + piece], key[-1])
                    off += piece
            r.result = r.out
        g.event = torch.cuda.Event()
        g.event.record(stream)

    def _run_staged(self, key, reqs, plans, stream, g) -> None:
        import torch

        spec = key[0] == "spectrogram"
        with torch.cuda.stream(self.upload):
            for r in reqs:
                if r.ready is not None:
                    self.upload.wait_event(r.ready)
                if getattr(r.data, "is_cuda", False):
                    r.data.record_stream(self.upload)
            if spec:
                fr, bins = reqs[0].out_shape()
                src = self._alloc((len(reqs), key[1]), torch.float32)
                dst = self._alloc((len(reqs), fr, bins), torch.float32)
                for i, r in enumerate(reqs):
                    src[i].copy_(r.data, non_blocking=True)
                g.buffers = [src, dst]
            else:
                rows = sum(r.rows() for r in reqs)
                shape = (rows, key[1]) if key[0] == "fft1d" else (rows, key[1], key[2])
                src = dst = self._alloc(shape, torch.complex64)
                g.buffers = [src]
                off = 0
                for r in reqs:
                    n = r.rows()
                    (src[off : off + n] if key[0] == "fft1d" else src[off]).copy_(r.data, non_blocking=True)
                    off += n
            uploaded = torch.cuda.Event()
            uploaded.record(self.upload)
        stream.wait_event(uploaded)
        if spec:
            for i in range(len(reqs)):
                plans[1](stream, dst[i], src[i])
        else:
            off = 0
            for piece in binary_pieces(rows):
                view = src[off : off + piece]
                plans[piece](stream, view, view, key[-1])
                off += piece
        computed = torch.cuda.Event()
        computed.record(stream)
        self.download.wait_event(computed)
        with torch.cuda.stream(self.download):
            off = 0
            for i, r in enumerate(reqs):
                if spec:
                    part = dst[i]
                else:
                    n = r.rows()
                    part = dst[off : off + n] if key[0] == "fft1d" else dst[off]
                    off += n
                r.result = r.out
                if r.result is None:
                    r.result = torch.empty(tuple(part.shape), dtype=part.dtype, pin_memory=True)
                elif getattr(r.result, "is_cuda", False):
                    r.result.record_stream(self.download)
                r.result.copy_(part, non_blocking=True)
            g.event = torch.cuda.Event()
            g.event.record(self.download)

    def _retire(self) -> None:
        now = None
        for d in self._inflight:
            while d and (d[0].event is None or d[0].event.query()):
                g = d.popleft()
                now = time.perf_counter() if now is None else now
                if g.error is not None:
                    self._fail(g.requests, g.error)
                else:
                    for r in g.requests:
                        r.finished, r.done, r.status = now, True, "done"
                    self.completed += len(g.requests)
                self._staged -= g.bytes
                g.buffers = []

    # -- driving -------------------------------------------------------------------
    def drain(self) -> None:
        """Run until every submitted request is finished."""
        while self.pending:
            if not self.step():
                time.sleep(20e-6)

    def run(self, requests, offsets=None) -> float:
        """Serve ``requests`` arriving at ``offsets`` seconds from now (all at once by
        default); returns the wall time until the last one finished."""
        order = sorted(range(len(requests)), key=lambda i: 0.0 if offsets is None else offsets[i])
        t0 = time.perf_counter()
        k = 0
        while k < len(order) or self.pending:
            now = time.perf_counter()
            while k < len(order) and (offsets is None or t0 + offsets[order[k]] <= now):
                i = order[k]
                self.submit(requests[i], now=t0 + (0.0 if offsets is None else offsets[i]))
                k += 1
            if not self.step():
                time.sleep(20e-6)
        return time.perf_counter() - t0


def serve_plain(requests, device=None, offsets=None, cache=None, cache_bytes: int = 60 << 30) -> float:
    """The per-call form: each request alone, in arrival order, with a plan compiled for
    its exact shape (as a caller of the reference compiles one computation per array
    shape), copied in, transformed, copied out and waited for before the next one.
    Returns the wall time; per-request times are recorded as for the server."""
    import torch

    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    cache = collections.OrderedDict() if cache is None else cache
    order = sorted(range(len(requests)), key=lambda i: 0.0 if offsets is None else offsets[i])
    t0 = time.perf_counter()
    for i in order:
        r = requests[i]
        r.arrival = t0 + (0.0 if offsets is None else offsets[i])
        now = time.perf_counter()
        if now < r.arrival:
            time.sleep(r.arrival - now)
        r.launched = time.perf_counter()
        k = (r.key(), tuple(r.data.shape))
        cc = cache.get(k)
        if cc is None:
            if r.kind == "spectrogram":
                comp = _spectrogram(r.data.shape[0], r.nfft, r.hop)
            else:
                comp = FFT(r.data, axes=(1,) if r.kind == "fft1d" else (0, 1))
            cc = cache[k] = comp.compile(device)
            held = sum(c._runner.plan.device_bytes for c in cache.values())
            while held > cache_bytes and len(cache) > 1:
                _, old = cache.popitem(last=False)
                held -= old._runner.plan.device_bytes
                old._runner.plan.close()
        else:
            cache.move_to_end(k)
        if r.data.is_cuda:
            # device-resident request: transform straight into its output
            x = r.data
            y = r.out if r.out is not None and r.out.is_cuda else None
        else:
            x = r.data.to(device)
            y = None
        if y is None:
            y = torch.empty(r.out_shape(), dtype=torch.float32, device=device) if r.kind == "spectrogram" else x
        if r.kind == "spectrogram":
            cc(None, y, x)
        else:
            cc(None, y, x, int(r.inverse))
        if r.out is not None:
            if r.out is not y:
                r.out.copy_(y)
            torch.cuda.current_stream(device).synchronize()
            r.result = r.out
        else:
            r.result = y.cpu()
        r.finished = time.perf_counter()
        r.done = True
    return time.perf_counter() - t0
