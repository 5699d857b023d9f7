"""The C ABI library: it loads without a GPU, exports every entry point the header declares,
and the ctypes mirror of each struct matches the C layout (checked by compiling the header)."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from paulistrings_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        names += re.findall(r"^[A-Za-z_][A-Za-z0-9_ \*]*?\b(ps_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_is_built_and_loads():
    L = _lib.lib()
    assert L.ps_abi_version() == 1


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 17
    for name in names:
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
    assert set(names) == set(_lib.EXPORTED)


def test_checked_build_exports_the_same_symbols():
    path = _lib.library_path(checked=True)
    if not path.exists():
        pytest.skip("checked build not present")
    L = ctypes.CDLL(str(path))
    for name in declared_functions():
        assert hasattr(L, name)


def test_device_count_is_safe_without_a_gpu():
    assert _lib.device_count() >= 0


def test_ctypes_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    checks = {
        "ps_keep_node": _lib.KeepNode,
        "ps_pass": _lib.Pass,
        "ps_policy": _lib.Policy,
        "ps_channel": _lib.Channel,
        "ps_table_entry": _lib.TableEntry,
        "ps_table": _lib.Table,
        "ps_layer_stats": _lib.LayerStats,
        "ps_run_stats": _lib.RunStats,
        "ps_kernel_profile": _lib.KernelProfile,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT / "include" / "paulistrings_b200.h"}"',
             "int main(void) {"]
    for cname, cls in checks.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {l.split()[0]: int(l.split()[-1]) for l in out if l.strip()}
    for cname, cls in checks.items():
        assert got[cname] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[f"{cname}.{fname}"] == getattr(cls, fname).offset, f"{cname}.{fname}"
