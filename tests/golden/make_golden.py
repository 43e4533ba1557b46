"""Generate golden fixtures from reikna's own FFT planner code.

reikna itself cannot be imported in this environment (its GPU backend grunnur,
Mako and PyOpenCL are not installed), but its planner is pure Python.  This script
parses ``reikna/fft/fft.py`` and ``reikna/helpers.py`` from a reikna checkout, executes
the planner functions and classes with a stub device description, and records:

* ``get_radix_array`` / ``get_global_radix_info`` for every power of two up to 2^24,
* ``get_kweights`` (Bluestein kernel weights) for several (N, M) pairs,
* the kernel chain ``FFT._build_plan`` would build (``get_fft_kernels`` plus the
  local-size fallback of ``_build_limited_plan``) for the benchmark shapes and the
  shapes of reikna's own tests, with ``prepare_for`` launch geometry.

Stub device (NVIDIA-like): max_total_local_size 1024, local_mem_size 49152,
local_mem_banks 32, align_words(word) = 128 // word.

Usage: python tests/golden/make_golden.py /path/to/reikna  (writes next to this file)
"""

from __future__ import annotations

import ast
import json
import sys
import types
from pathlib import Path

import numpy

HERE = Path(__file__).resolve().parent


def _extract(path: Path, names: set[str]) -> ast.Module:
    tree = ast.parse(path.read_text())
    body = [ast.ImportFrom(module="__future__", names=[ast.alias(name="annotations")], level=0)]
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            body.append(node)
        elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in names for t in node.targets):
            body.append(node)
    mod = ast.Module(body=body, type_ignores=[])
    ast.fix_missing_locations(mod)
    return mod


class _Stub:
    def __getattr__(self, name):
        return lambda *a, **k: None


class VirtualSizeError(Exception):
    pass


class DeviceParams:
    max_total_local_size = 1024
    local_mem_size = 49152
    local_mem_banks = 32

    @staticmethod
    def align_words(word_size: int) -> int:
        return 128 // word_size


def load_reference(root: Path) -> dict:
    import functools

    helpers_ns: dict = {"numpy": numpy, "functools": functools}
    exec(
        compile(
            _extract(root / "reikna" / "helpers.py", {"product", "min_blocks", "log2", "bounding_power_of_2"}),
            "reikna/helpers.py",
            "exec",
        ),
        helpers_ns,
    )
    helpers = types.SimpleNamespace(**{k: helpers_ns[k] for k in ("product", "min_blocks", "log2", "bounding_power_of_2")})
    ns: dict = {
        "numpy": numpy,
        "helpers": helpers,
        "dtypes": _Stub(),
        "functions": _Stub(),
        "VirtualSizeError": VirtualSizeError,
        "Any": object,
    }
    names = {
        "MAX_RADIX",
        "get_radix_array",
        "get_global_radix_info",
        "get_padding",
        "get_local_memory_size",
        "get_kweights",
        "get_common_kwds",
        "LocalFFTKernel",
        "GlobalFFTKernel",
        "get_fft_1d_kernels",
        "get_fft_kernels",
    }
    exec(compile(_extract(root / "reikna" / "fft" / "fft.py", names), "reikna/fft/fft.py", "exec"), ns)
    return ns


def build_chain(ns: dict, shape, dtype, axes) -> dict:
    """FFT._build_plan's kernel search (reikna/fft/fft.py:664-756) without codegen."""
    dp = DeviceParams()
    limit = dp.max_total_local_size
    while limit >= 1:
        kernels = ns["get_fft_kernels"](tuple(shape), numpy.dtype(dtype), tuple(axes), dp, limit)
        recs = []
        try:
            for k in kernels:
                ls = dp.max_total_local_size
                while ls >= 1:
                    try:
                        gsize, lsize, kwds = k.prepare_for(ls)
                    except VirtualSizeError:
                        if isinstance(k, ns["GlobalFFTKernel"]):
                            ls //= 2
                            continue
                        raise
                    break
                rec = dict(
                    kind="local" if isinstance(k, ns["LocalFFTKernel"]) else "global",
                    output_shape=list(k.output_shape),
                    gsize=int(gsize),
                    lsize=int(lsize),
                    fft_size=int(kwds["fft_size"]),
                    fft_size_real=int(kwds["fft_size_real"]),
                    reverse_direction=bool(kwds["reverse_direction"]),
                    pad_in=bool(kwds["pad_in"]),
                    unpad_out=bool(kwds["unpad_out"]),
                    takes_kweights=bool(kwds["takes_kweights"]),
                    has_kweights=k.kweights is not None,
                )
                if rec["kind"] == "local":
                    rec["radix"] = [int(r) for r in kwds["radix_arr"]]
                    rec["pass_num"] = 0
                else:
                    rec["radix"] = [int(kwds["radix"])]
                    rec["radix1"] = int(kwds["radix1"])
                    rec["radix2"] = int(kwds["radix2"])
                    rec["pass_num"] = int(kwds["pass_num"])
                recs.append(rec)
        except VirtualSizeError:
            limit //= 2
            continue
        return dict(local_kernel_limit=limit, kernels=recs)
    raise RuntimeError("no plan")


CHAIN_CASES = [
    ((64, 4096), "complex64", (1,)),
    ((256, 256, 256), "complex64", (0, 1, 2)),
    ((128, 128, 128), "complex128", (0, 1, 2)),
    ((1000, 3001), "complex64", (1,)),
    ((1000, 1000), "complex64", (0, 1)),
    ((16384, 1024), "complex64", (1,)),
    ((2**20,), "complex64", (0,)),
    ((65521,), "complex64", (0,)),
    ((3, 255, 7), "complex64", (2, 0)),
    ((17, 200, 131), "complex64", (1, 0)),
    ((7, 1000, 11), "complex64", (1, 2)),
    ((15, 900, 57), "complex64", (2, 0, 1)),
    ((1, 2**15, 3), "complex64", (1,)),
    ((4, 127, 64), "complex64", (1,)),
    ((1000, 501), "complex64", (0,)),
]

KW_CASES = [(7, 16), (100, 256), (127, 256), (1000, 2048)]


def main(argv: list[str]) -> int:
    if len(argv) != 2:
        print(f"usage: python {Path(argv[0]).name} <path of a fjarri/reikna checkout>", file=sys.stderr)
        return 2
    root = Path(argv[1])
    ns = load_reference(root)
    pow2 = [2**k for k in range(1, 25)]
    radix = {
        str(s): {
            "radix_array": ns["get_radix_array"](s) if s <= 2**20 else None,
            "radix_array_max": ns["get_radix_array"](s, use_max_radix=True) if s <= 2**20 else None,
            "global": [list(map(int, x)) for x in ns["get_global_radix_info"](s)],
        }
        for s in pow2
    }
    chains = [
        dict(shape=list(shape), dtype=dt, axes=list(axes), **build_chain(ns, shape, dt, axes))
        for shape, dt, axes in CHAIN_CASES
    ]
    (HERE / "planner.json").write_text(json.dumps({"radix": radix, "chains": chains}, indent=1))
    arrays = {}
    for n, m in KW_CASES:
        kw = ns["get_kweights"](n, m)
        arrays[f"kw_{n}_{m}"] = kw.astype(numpy.complex128)
    numpy.savez_compressed(HERE / "kweights.npz", **arrays)
    print("wrote", HERE / "planner.json", HERE / "kweights.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
