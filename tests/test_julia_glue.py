"""The Julia glue's ccalls agree with include/epb200.h (no Julia needed).

For every `ccall((:epb_..., LIB[]), Cint, (types...), ...)` in julia/ElectronPhononB200.jl, the named
entry point is declared in the header with the same number of parameters, and each argument type has
the header parameter's kind: a pointer (Ptr, CuPtr, Ref, Cstring) for a C pointer, an integer or float
type of the same width for a C scalar.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "electronphonon.jl_b200", "julia", "ElectronPhononB200.jl")
HDR = os.path.join(ROOT, "include", "epb200.h")


def split_top(s):
    """Split at commas outside brackets / braces / parentheses."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def header_protos():
    txt = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"EPB_API\s+[\w\s\*]+?\b(epb_\w+)\s*\(([^;]*?)\)\s*;", txt, flags=re.S):
        params = [p for p in split_top(" ".join(m.group(2).split())) if p and p != "void"]
        protos[m.group(1)] = params
    return protos


def ccalls():
    txt = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(\(:(epb_\w+),", txt):
        i, depth = m.start() + len("ccall"), 0
        for j in range(i, len(txt)):  # the whole ccall( ... )
            depth += txt[j] == "("
            depth -= txt[j] == ")"
            if depth == 0:
                break
        args = split_top(txt[i + 1:j])
        calls.append((m.group(1), split_top(args[2].strip()[1:-1])))
    return calls


def c_kind(param):
    t = param.rsplit(None, 1)[0] if "*" not in param.split()[-1] else param
    if "*" in param:
        return "ptr"
    t = param.split()[:-1] if len(param.split()) > 1 else param.split()
    t = " ".join(w for w in t if w != "const")
    return {"int64_t": "i64", "uint64_t": "i64", "int": "i32", "int32_t": "i32", "double": "f64",
            "char": "i8", "float": "f32"}.get(t, t)


def jl_kind(t):
    t = t.strip()
    if t.startswith(("Ptr{", "CuPtr{", "Ref{")) or t in ("Cstring", "Ptr"):
        return "ptr"
    return {"Int64": "i64", "UInt64": "i64", "Cint": "i32", "Int32": "i32", "Float64": "f64", "Cdouble": "f64",
            "Cchar": "i8", "UInt8": "i8", "Float32": "f32"}.get(t, t)


def test_every_ccall_matches_its_prototype():
    protos = header_protos()
    calls = ccalls()
    assert len(calls) >= 20
    for name, types in calls:
        assert name in protos, f"{name} is not declared in the header"
        params = protos[name]
        assert len(types) == len(params), f"{name}: {len(types)} argument types, header has {len(params)}"
        for k, (t, p) in enumerate(zip(types, params)):
            assert jl_kind(t) == c_kind(p), f"{name} argument {k + 1}: Julia {t} vs C {p}"


JL_SIZE = {"Int64": 8, "UInt64": 8, "Float64": 8, "Cint": 4, "Int32": 4, "Cdouble": 8}


def jl_size_align(t):
    t = t.strip()
    if t in JL_SIZE:
        return JL_SIZE[t], JL_SIZE[t]
    if t.startswith("Ptr{") or t.startswith("CuPtr{"):
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", t)
    if m:
        sz, al = jl_size_align(m.group(2))
        return int(m.group(1)) * sz, al
    raise AssertionError(f"no C layout known for Julia type {t}")


def jl_structs():
    """{C struct name: [(field, offset), ..., ('size', n)]} of the `struct X  # epb_name` mirrors."""
    txt = open(JL).read()
    out = {}
    for m in re.finditer(r"^struct (\w+)\s*#\s*(epb_\w+)[^\n]*\n(.*?)^end", txt, flags=re.S | re.M):
        off, align, fields = 0, 1, []
        for line in m.group(3).splitlines():
            f = re.match(r"\s*(\w+)::(.+?)\s*$", line)
            if not f:
                continue
            sz, al = jl_size_align(f.group(2))
            off = (off + al - 1) // al * al
            fields.append((f.group(1), off))
            off += sz
            align = max(align, al)
        fields.append(("size", (off + align - 1) // align * align))
        out[m.group(2)] = fields
    return out


def test_julia_struct_mirrors_match_the_header(tmp_path):
    import shutil
    import subprocess

    import pytest

    if shutil.which("gcc") is None:
        pytest.skip("needs gcc")
    structs = jl_structs()
    assert {"epb_bte_params", "epb_tiled_info", "epb_outer_q_params", "epb_kbatch_payload",
            "epb_outer_q_calc"} <= set(structs)
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "epb200.h"', 'int main(void) {']
    for cname, fields in structs.items():
        for f, _ in fields:
            expr = f"sizeof({cname})" if f == "size" else f"offsetof({cname}, {f})"
            lines.append(f'  printf("{cname} {f} %zu\\n", {expr});')
    lines += ['  return 0;', '}']
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, f, v = line.split()
        got[(c, f)] = int(v)
    for cname, fields in structs.items():
        for f, off in fields:
            assert got[(cname, f)] == off, (cname, f, off, got[(cname, f)])
