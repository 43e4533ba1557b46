"""Autotuner for a single computation: kernel shapes chosen by timing them.

reikna picks its kernel parameters by rules (radix tables, work-group sizes from the
device limits, reikna/fft/fft.py:24-213 and :699-756, halving the local size until a
kernel compiles).  Here the planner's rules give a default; the choices below are
measured on the caller's own arguments and the fastest is kept:

* tile shape of two innermost power-of-two axes: one clustered plane pass
  (16-CTA clusters, 16 rows a CTA), the same on twice-as-wide clusters
  (``FLAG_PLANE_WIDE``), a row pass and a column pass in one plane-ordered persistent
  launch (``FLAG_PAIR``), or separate line passes (``FLAG_NO_PLANE``);
* operand staging: persistent TMA-fed line passes or plain per-tile loads
  (``FLAG_NO_TMA``);
* threads per transform and radix plan of 8192-point Bluestein lines: one CTA of 256
  threads with 32 elements a thread (the default), 16 on 512 (``FLAG_R16``), or a
  two-CTA cluster a line, each CTA one half of the padded spectrum
  (``FLAG_BLUE_PAIR``);
* Bluestein in one fused pass or as separate FFT passes (``FLAG_NO_BLUE1``);
* a real signal's transform as the half-length FFT of sample pairs or at full length
  (``FLAG_NO_HALF``);
* with ``allow_split``, the tensor-core split-precision stages (``FLAG_SPLIT_TC``,
  a different accuracy: opt-in).

Choices are cached in JSON (``RK_AUTOTUNE_CACHE``, default
``~/.cache/reikna_b200/autotune.json``) keyed by the computation's native descriptor.
"""

from __future__ import annotations

import hashlib

from . import _native as N
from .batch import _load_cache, _store_cache

_VERSION = b"fft-tune-1"


def candidates(comp, allow_split: bool = False) -> list[int]:
    """Plan-flag sets worth timing for ``comp`` (an FFT), the default first."""
    passes = comp.describe(0)["passes"]
    out = [0]
    if any(p["kind"] == "line" and p["var"] == 0 for p in passes):
        out.append(N.FLAG_NO_TMA)
    if any(p["kind"] == "plane" for p in passes):
        out += [N.FLAG_NO_PLANE, N.FLAG_PLANE_WIDE, N.FLAG_PAIR]
    blue = [p for p in passes if p["var"] & 15 == 1]
    if blue:
        out.append(N.FLAG_NO_BLUE1)
        if any(p["L"] == 8192 and p["mode"] == "pos" and p["var"] & 15 == 1 for p in blue):
            out += [N.FLAG_R16, N.FLAG_BLUE_PAIR]
    if any(p["note"] == "half" for p in passes):
        out.append(N.FLAG_NO_HALF)
    if allow_split and any(p["kind"] == "line" and p["L"] == 1024 and p["mode"] == "pos" and p["var"] == 0
                           for p in passes):
        out.append(N.FLAG_SPLIT_TC)
    return out


def _key(comp, allow_split: bool) -> str:
    h = hashlib.sha256(_VERSION + (b"split" if allow_split else b""))
    h.update(bytes(comp.native_descriptor(0)[0]))
    return h.hexdigest()[:32]


def tune(comp, args, device=None, reps: int = 20, allow_split: bool = False, use_cache: bool = True) -> dict:
    """Time every candidate of ``comp`` on ``args`` (the positional arguments its
    compiled callable takes); returns {"flags": best, "tried": [...], "cached": bool}."""
    import torch

    key = _key(comp, allow_split)
    if use_cache:
        hit = _load_cache().get(key)
        if hit is not None:
            return {"cached": True, **hit}
    tried = []
    best = None
    for flags in candidates(comp, allow_split):
        try:
            cc = comp.compile(device, flags=flags)
        except (N.NativeError, NotImplementedError, ValueError):
            continue
        for _ in range(3):
            cc(None, *args)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            cc(None, *args)
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e) / reps
        tried.append({"flags": flags, "ms": ms})
        if best is None or ms < best[0]:
            best = (ms, flags)
    if best is None:
        raise N.NativeError(N.ERR_UNSUPPORTED, "no candidate plan could run")
    entry = {"flags": best[1], "ms": best[0], "tried": tried}
    if use_cache:
        _store_cache(key, entry)
    return {"cached": False, **entry}


def compile_tuned(comp, args, device=None, **kw):
    """``comp.compile`` with the plan flags ``tune`` picks for ``args``; the result
    carries the tuning record in ``.tuning``."""
    rec = tune(comp, args, device, **kw)
    cc = comp.compile(device, flags=rec["flags"])
    cc.tuning = rec
    return cc
