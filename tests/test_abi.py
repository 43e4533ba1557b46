"""The C-ABI library: loads without a GPU, exports every declared symbol, plans on CPU."""

import ctypes
import re
from pathlib import Path

import pytest

from reikna_b200 import _native as N

HEADER = Path(__file__).resolve().parent.parent / "include" / "reikna_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return re.findall(r"RK_API\s+[\w\s\*]+?\b(rk_\w+)\s*\(", text)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "rk_fft_plan_create" in names and "rk_fft_execute" in names
    assert set(names) == set(N.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = __import__("subprocess").run(["nm", "-D", "--defined-only", str(N.library_path())], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (rk_\w+)", out.stdout))
    assert set(declared_functions()) <= exported


def test_abi_struct_sizes():
    eb, db = ctypes.c_int64(), ctypes.c_int64()
    assert N.lib().rk_abi_sizes(ctypes.byref(eb), ctypes.byref(db)) == 0
    assert eb.value == ctypes.sizeof(N.Edge)
    assert db.value == ctypes.sizeof(N.FftDesc)


def test_version():
    assert b"sm_100a" in N.lib().rk_version()


def test_describe_bench_configs():
    d = N.describe(N.desc(N.FMT_C64, (64, 4096), (1,)))
    assert [p["L"] for p in d["passes"]] == [4096]
    d = N.describe(N.desc(N.FMT_C64, (1000, 3001), (1,)))
    assert d["passes"][0]["note"] == "bluestein-fused" and d["passes"][0]["L"] == 8192
    assert d["bluestein"] == [{"axis": 1, "N": 3001, "M": 8192}]
    d = N.describe(N.desc(N.FMT_C64, (2**20,), (0,)))
    assert [p["note"] for p in d["passes"]] == ["fourstep-A", "fourstep-B"]
    d = N.describe(N.desc(N.FMT_C64, (65521,), (0,)))
    assert len(d["passes"]) == 4 and d["bluestein"][0]["M"] == 131072


def test_describe_3d_uses_at_most_three_passes():
    d = N.describe(N.desc(N.FMT_C64, (256, 256, 256), (0, 1, 2)))
    assert 1 <= len(d["passes"]) <= 3
    assert d["passes"][0]["in"] == "input" and d["passes"][-1]["out"] == "output"


def test_describe_trivial_is_one_copy_pass():
    d = N.describe(N.desc(N.FMT_C64, (128, 1, 1, 128), (1, 2)))
    assert [p["note"] for p in d["passes"]] == ["copy"]


@pytest.mark.parametrize(
    "shape,axes,msg",
    [
        ((8,), (1,), "axis out of range"),
        ((8, 8), (0, 0), "repeated axis"),
        ((0, 8), (1,), "shape entries must be positive"),
    ],
)
def test_invalid_descriptors(shape, axes, msg):
    d = N.desc(N.FMT_C64, tuple(max(1, s) for s in shape), ())
    d.naxes = len(axes)
    for i, a in enumerate(axes):
        d.axes[i] = a
    for i, s in enumerate(shape):
        d.shape[i] = s
    with pytest.raises(ValueError, match=msg):
        N.describe(d)


def test_non_complex_dtype_rejected():
    d = N.desc(N.FMT_C64, (16,), (0,))
    d.dtype = N.FMT_F32
    with pytest.raises(ValueError, match="complex dtype"):
        N.describe(d)
