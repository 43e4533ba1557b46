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
buffer per group.
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

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


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
        with torch.cuda.device(self.device):
            self.streams = [torch.cuda.Stream(self.device) for _ in range(streams)]
            self.upload = torch.cuda.Stream(self.device)
            self.download = torch.cuda.Stream(self.device)
        self.plans = PlanCache(self.device, plan_budget)
        self._class_stream = {}
        self._waiting = collections.OrderedDict()  # class key -> deque of requests
        self._inflight = [collections.deque() for _ in range(streams)]
        self._staged = 0
        self.groups = 0
        self.completed = 0

    # -- intake ------------------------------------------------------------------
    def submit(self, req: FFTRequest, now: float | None = None) -> FFTRequest:
        key = req.key()
        req.arrival = time.perf_counter() if now is None else now
        self._waiting.setdefault(key, collections.deque()).append(req)
        return req

    @property
    def pending(self) -> int:
        return sum(len(q) for q in self._waiting.values()) + sum(
            len(g.requests) for d in self._inflight for g in d
        )

    # -- scheduling ----------------------------------------------------------------
    def stream_of(self, key) -> int:
        s = self._class_stream.get(key)
        if s is None:
            s = self._class_stream[key] = len(self._class_stream) % len(self.streams)
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
        Returns the number of groups launched."""
        self._retire()
        launched = 0
        while True:
            key = self._next_class()
            if key is None:
                break
            s = self.stream_of(key)
            reqs = self._take(key)
            need = self.group_bytes(reqs)
            if self._staged and self._staged + need > self.memory_budget:
                # wait for memory: put the requests back at the head of their queue
                self._waiting[key].extendleft(reversed(reqs))
                break
            self._launch(key, reqs, s, need)
            launched += 1
        return launched

    def _launch(self, key, reqs, s: int, need: int) -> None:
        """Three-stage pipeline of one group: host-to-device copies on the upload
        stream, the transforms on the class's compute stream, device-to-host copies on
        the download stream, chained by events.  Uploads of later groups run while
        earlier groups compute and download (the link carries both directions at once)."""
        import torch

        stream = self.streams[s]
        now = time.perf_counter()
        g = _Group(key, reqs, s, need)
        spec = key[0] == "spectrogram"
        if all(r.data.is_cuda and r.out is not None and r.out.is_cuda for r in reqs):
            # device-resident requests with device outputs: no staging, each request
            # is transformed from its input straight into its output
            g.bytes = 0
            with torch.cuda.device(self.device):
                for r in reqs:
                    if spec:
                        self.plans.get(key, 1)(stream, r.out, r.data)
                    elif key[0] == "fft2d":
                        self.plans.get(key, 1)(stream, r.out[None], r.data[None], key[-1])
                    else:
                        off = 0
                        for piece in binary_pieces(r.rows()):
                            self.plans.get(key, piece)(stream, r.out[off : off + piece], r.data[off : off + piece], key[-1])
                            off += piece
                    r.result = r.out
                g.event = torch.cuda.Event()
                g.event.record(stream)
            for r in reqs:
                r.launched = now
            self._inflight[s].append(g)
            self.groups += 1
            return
        with torch.cuda.device(self.device):
            with torch.cuda.stream(self.upload):
                if spec:
                    fr, bins = reqs[0].out_shape()
                    src = torch.empty((len(reqs), key[1]), dtype=torch.float32, device=self.device)
                    dst = torch.empty((len(reqs), fr, bins), dtype=torch.float32, device=self.device)
                    for i, r in enumerate(reqs):
                        src[i].copy_(r.data, non_blocking=True)
                    g.buffers = [src, dst]
                else:
                    rows = sum(r.rows() for r in reqs)
                    shape = (rows, key[1]) if key[0] == "fft1d" else (rows, key[1], key[2])
                    src = dst = torch.empty(shape, dtype=torch.complex64, device=self.device)
                    off = 0
                    for r in reqs:
                        n = r.rows()
                        (src[off : off + n] if key[0] == "fft1d" else src[off]).copy_(r.data, non_blocking=True)
                        off += n
                    g.buffers = [src]
                uploaded = torch.cuda.Event()
                uploaded.record(self.upload)
            stream.wait_event(uploaded)
            if spec:
                cc = self.plans.get(key, 1)
                for i in range(len(reqs)):
                    cc(stream, dst[i], src[i])
            else:
                off = 0
                for piece in binary_pieces(rows):
                    view = src[off : off + piece]
                    self.plans.get(key, piece)(stream, view, view, key[-1])
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
                    r.result.copy_(part, non_blocking=True)
                g.event = torch.cuda.Event()
                g.event.record(self.download)
        for r in reqs:
            r.launched = now
        self._staged += need
        self._inflight[s].append(g)
        self.groups += 1

    def _retire(self) -> None:
        now = None
        for d in self._inflight:
            while d and d[0].event.query():
                g = d.popleft()
                now = time.perf_counter() if now is None else now
                for r in g.requests:
                    r.finished = now
                    r.done = True
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
