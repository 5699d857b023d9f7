"""The Rust binding that INTEGRATION.md tells a maintainer to copy must have the C layout.

Every ``#[repr(C)] pub struct Ps...`` in its Rust block is laid out here by the repr(C) rules
(fields in order, each at the next multiple of its alignment, the size rounded up to the
largest alignment), and each size and field offset is compared with ``sizeof`` / ``offsetof``
of the ``ps_...`` twin compiled from ``include/paulistrings_b200.h``.  Every ``pub fn ps_...``
it declares must be a function the header declares.  Runs on the CPU (gcc only).
"""

import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
DOC = ROOT / "INTEGRATION.md"
HEADER = ROOT / "include" / "paulistrings_b200.h"

PRIM = {"i8": 1, "u8": 1, "i16": 2, "u16": 2, "i32": 4, "u32": 4, "f32": 4, "i64": 8, "u64": 8, "f64": 8,
        "usize": 8, "isize": 8}


def rust_block():
    text = DOC.read_text()
    m = re.search(r"```rust\n(.*?)```", text, flags=re.S)
    assert m, "no Rust block in INTEGRATION.md"
    return m.group(1)


def parse_structs(block):
    structs = {}
    for m in re.finditer(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}", block, flags=re.S):
        name, body = m.group(1), m.group(2)
        fields = []
        for f in re.finditer(r"(?:pub\s+)?(\w+)\s*:\s*(\[[^\]]+\]|\*(?:const|mut)\s+\w+|\w+)", body):
            fields.append((f.group(1), f.group(2).strip()))
        structs[name] = fields
    return structs


def layout(structs, name, memo):
    """(size, align, {field: offset}) of a repr(C) struct."""
    if name in memo:
        return memo[name]

    def type_info(t):
        t = t.strip()
        if t.startswith("["):
            inner, count = t[1:-1].rsplit(";", 1)
            s, a = type_info(inner)
            return s * int(count), a
        if t.startswith("*"):
            return 8, 8
        if t in PRIM:
            return PRIM[t], PRIM[t]
        s, a, _ = layout(structs, t, memo)
        return s, a

    off, align, offsets = 0, 1, {}
    for fname, ftype in structs[name]:
        s, a = type_info(ftype)
        off = (off + a - 1) // a * a
        offsets[fname] = off
        off += s
        align = max(align, a)
    size = (off + align - 1) // align * align
    memo[name] = (size, align, offsets)
    return memo[name]


def c_name(rust_name):
    return "ps" + re.sub(r"([A-Z])", lambda m: "_" + m.group(1).lower(), rust_name[2:])


def test_rust_mirror_matches_the_c_layout(tmp_path):
    structs = parse_structs(rust_block())
    mirrored = {k: v for k, v in structs.items() if not (len(v) == 1 and v[0][0] == "_p")}
    for needed in ("PsPass", "PsPolicy", "PsKeepNode", "PsChannel", "PsTable", "PsLayerStats", "PsScorerConfig"):
        assert needed in mirrored, f"INTEGRATION.md does not mirror {needed}"
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for rname, fields in mirrored.items():
        cn = c_name(rname)
        lines.append(f'printf("{rname} size %zu\\n", sizeof({cn}));')
        for fname, _ in fields:
            lines.append(f'printf("{rname}.{fname} %zu\\n", offsetof({cn}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "doc_layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "doc_layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {" ".join(l.split()[:-1]): int(l.split()[-1]) for l in out if l.strip()}
    memo = {}
    for rname, fields in mirrored.items():
        size, _, offsets = layout(structs, rname, memo)
        assert size == got[f"{rname} size"], f"{rname}: {size} bytes in INTEGRATION.md, {got[rname + ' size']} in C"
        for fname, _ in fields:
            assert offsets[fname] == got[f"{rname}.{fname}"], f"{rname}.{fname}"


def test_rust_mirror_declares_only_exported_functions():
    declared = set(re.findall(r"\b(ps_[a-z_0-9]+)\s*\(", HEADER.read_text()))
    bound = set(re.findall(r"pub fn (ps_[a-z_0-9]+)\s*\(", rust_block()))
    assert bound, "no functions in the Rust block"
    assert bound <= declared, sorted(bound - declared)
