"""The Julia binding (peakpatch.jl_b200/julia/PeakPatchB200.jl) against the C
header, without Julia: its structs must have the C structs' field order and
byte offsets, and every ccall must name an exported function with the
header's parameter count and compatible argument types.  CPU only."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

SHIM = os.path.join(ROOT, "peakpatch.jl_b200", "julia", "PeakPatchB200.jl")
HEADER = os.path.join(ROOT, "include", "ppb.h")

# Julia isbits types -> (size, alignment) under the C layout rules Julia uses
JL = {"Float64": (8, 8), "Float32": (4, 4), "Int64": (8, 8), "UInt64": (8, 8), "Int32": (4, 4), "UInt32": (4, 4),
      "Int8": (1, 1), "Ptr{Float32}": (8, 8), "Ptr{Cvoid}": (8, 8)}


def julia_struct(src, name):
    m = re.search(r"(?:mutable\s+)?struct\s+" + name + r"\s*\n(.*?)\nend", src, re.S)
    assert m, name
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("#")[0]
        for part in line.split(";"):
            part = part.strip()
            if not part:
                continue
            fname, ftype = [x.strip() for x in part.split("::")]
            nt = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", ftype)
            if nt:
                size, al = JL[nt.group(2)]
                fields.append((fname, int(nt.group(1)) * size, al))
            else:
                size, al = JL[ftype]
                fields.append((fname, size, al))
    off, out, maxal = 0, [], 1
    for fname, size, al in fields:
        off = (off + al - 1) // al * al
        out.append((fname, off))
        off += size
        maxal = max(maxal, al)
    return out, (off + maxal - 1) // maxal * maxal


def c_layout(tmp_path, struct, fields):
    prog = tmp_path / "lay.c"
    body = "".join(f'  printf("{f} %zu\\n", offsetof({struct}, {f}));\n' for f in fields)
    prog.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "ppb.h"\nint main(void) {{\n{body}'
                    f'  printf("SIZE %zu\\n", sizeof({struct}));\n  return 0;\n}}\n')
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    d = dict(zip(out[::2], map(int, out[1::2])))
    return d


@pytest.mark.parametrize("jl_name,c_name", [("TileParams", "ppb_tile_params"), ("HaloBuf", "ppb_halo_buf")])
def test_julia_structs_match_the_header(tmp_path, jl_name, c_name):
    src = open(SHIM).read()
    fields, size = julia_struct(src, jl_name)
    c = c_layout(tmp_path, c_name, [f for f, _ in fields])
    for f, off in fields:
        assert c[f] == off, (jl_name, f, off, c[f])
    assert c["SIZE"] == size


def _c_prototypes():
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(?:int32_t|void)\s+(ppb_\w+)\s*\(([^)]*)\)\s*;", txt):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(1)] = args
    return protos


# C parameter type -> Julia ccall argument types that pass it correctly
_SCALAR = {"int32_t": "Int32", "int64_t": "Int64", "uint64_t": "UInt64", "double": "Float64", "float": "Float32",
           "size_t": "Csize_t", "int8_t": "Int8", "char": "UInt8"}
_STRING = {"Cstring", "Ptr{UInt8}"}


def _compatible(cparam, jtype):
    ctype = re.sub(r"\bconst\b", "", cparam).strip()
    if "*" in ctype:
        inner = ctype.split("*")[0].strip()
        if jtype == "Ptr{Cvoid}":
            return True
        if inner == "char" and jtype in _STRING:
            return True
        if inner in _SCALAR:
            return jtype in (f"Ptr{{{_SCALAR[inner]}}}", f"Ref{{{_SCALAR[inner]}}}")
        return inner.startswith("ppb_") and jtype.startswith(("Ref{", "Ptr{"))   # a struct of the header
    return _SCALAR.get(ctype.split()[0]) == jtype


def test_julia_ccalls_match_the_header():
    protos = _c_prototypes()
    src = open(SHIM).read()
    calls = re.findall(r"ccall\(\(:(ppb_\w+),\s*libppb\),\s*Int32,\s*\((.*?)\),", src, re.S)
    assert len(calls) >= 15
    for name, types in calls:
        assert name in protos, name
        jt = [t.strip() for t in re.split(r",(?![^{]*\})", types.replace("\n", " ")) if t.strip()]
        assert len(jt) == len(protos[name]), (name, len(jt), len(protos[name]))
        for ct, j in zip(protos[name], jt):
            assert _compatible(ct, j), (name, ct, j)
