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


# ---------------------------------------------------------------------------------------------
# Dispatch: the glue's methods must be the ones Julia selects at the reference's own call sites.
# tests/golden/julia_call_sites.json (made by tests/golden/make_julia_call_sites.py from the reference)
# lists every device-path call of an overridden method with each argument's kind; the CUDA extension's
# method signatures are listed there too. CUDA.jl's array aliases order as
#   CuArray < DenseCuArray (adds contiguous views, reshapes) < StridedCuArray (adds strided views)
#   < AnyCuArray (adds any wrapper, e.g. a reshape of a view) < untyped.
import json  # noqa: E402

GOLD = os.path.join(ROOT, "tests", "golden", "julia_call_sites.json")
ALIAS = {"CuArray": ("CuArray", None), "CuMatrix": ("CuArray", 2), "CuVector": ("CuArray", 1),
         "DenseCuArray": ("DenseCuArray", None), "DenseCuMatrix": ("DenseCuArray", 2),
         "DenseCuVector": ("DenseCuArray", 1), "StridedCuArray": ("StridedCuArray", None),
         "StridedCuMatrix": ("StridedCuArray", 2), "StridedCuVector": ("StridedCuArray", 1),
         "AnyCuArray": ("AnyCuArray", None), "AnyCuMatrix": ("AnyCuArray", 2), "AnyCuVector": ("AnyCuArray", 1)}
FAMILY_OK = {"dev": {"CuArray", "DenseCuArray", "StridedCuArray", "AnyCuArray"},
             "dense": {"DenseCuArray", "StridedCuArray", "AnyCuArray"},
             "strided": {"StridedCuArray", "AnyCuArray"}, "rview": {"AnyCuArray"}}
ELT = {"Int": "Int64", "Complex{Float64}": "ComplexF64", "Complex{T}": "ComplexF64", "T": None}


def _norm_elt(e):
    e = e.strip()
    return ELT.get(e, e)


def _family(kind):
    if kind.startswith("dev:"):
        return "dev"
    if kind.startswith("view:"):
        return kind.split(":")[3]
    if kind.startswith("rview:"):
        return "rview"
    return kind


def accepts(decl, kind):
    """Does a Julia parameter declared `decl` (None = untyped) accept an argument of `kind`?"""
    if decl is None or decl == "Any":
        return True
    decl = decl.strip()
    m = re.fullmatch(r"Union\{(.*)\}", decl)
    if m:
        return any(accepts(d, kind) for d in split_top(m.group(1)))
    if kind == "nothing":
        return decl == "Nothing"
    if kind in ("char", "int", "any", "range", "host-kvec", "itp"):
        return {"char": {"Char"}, "int": {"Int", "Integer", "Int64"}, "itp": {
            "ElectronPhonon.BatchedWannierInterpolator", "BatchedWannierInterpolator"}}.get(kind, set()) >= {decl} \
            if kind in ("char", "int", "itp") else False
    m = re.fullmatch(r"(\w+)(?:\{(.*)\})?", decl)
    if not m or m.group(1) not in ALIAS:
        return False
    base, nd_alias = ALIAS[m.group(1)]
    params = split_top(m.group(2)) if m.group(2) else []
    elt = _norm_elt(params[0]) if params else None
    nd = int(params[1]) if len(params) > 1 else nd_alias
    fam = _family(kind)
    if fam not in FAMILY_OK or base not in FAMILY_OK[fam]:
        return False
    _, k_elt, k_nd = kind.split(":")[:3]
    return (elt is None or elt == _norm_elt(k_elt)) and (nd is None or nd == int(k_nd))


def glue_methods():
    """{name: [(positional [(name, decl)], keywords {name: decl})]} of `function ElectronPhonon.name(...)`."""
    txt = open(JL).read()
    out = {}
    for m in re.finditer(r"^function ElectronPhonon\.([\w!]+)\(", txt, flags=re.M):
        i, depth = m.end() - 1, 0
        for j in range(i, len(txt)):
            depth += txt[j] == "("
            depth -= txt[j] == ")"
            if depth == 0:
                break
        body = " ".join(txt[i + 1:j].split())
        pos_txt, _, kw_txt = body.partition(";")
        pos = []
        for p in split_top(pos_txt):
            nm, _, ty = p.partition("::")
            pos.append((nm.strip(), ty.strip() or None))
        kw = {}
        for p in split_top(kw_txt):
            lhs = p.split("=", 1)[0].strip()
            nm, _, ty = lhs.partition("::")
            kw[nm.strip()] = ty.strip() or None
        out.setdefault(m.group(1), []).append((pos, kw))
    return out


def _sig_accepts(sig, pos_kinds, kw_kinds):
    pos, kw = sig
    if len(pos) != len(pos_kinds):
        return False
    if not all(accepts(d, k) for (_, d), k in zip(pos, pos_kinds)):
        return False
    return all(name in kw and accepts(kw[name], k) for name, k in kw_kinds.items())


def test_call_site_fixture_matches_the_reference():
    import pytest

    if not os.path.isdir("/root/reference"):
        pytest.skip("reference sources not present")
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_julia_call_sites as M

    gold = json.load(open(GOLD))
    assert M.build("/root/reference") == gold["sites"]
    assert M.ext_methods("/root/reference") == gold["ext_methods"]


def test_glue_methods_dispatch_at_every_reference_call_site():
    """Each device-path call of an overridden method in the reference (views included) matches a glue method
    by its declared types, so the reference loop reaches the library instead of the generic CPU method."""
    gold = json.load(open(GOLD))
    glue = glue_methods()
    assert len(gold["sites"]) >= 12
    for s in gold["sites"]:
        sigs = glue.get(s["method"])
        assert sigs, f"no glue method {s['method']} ({s['file']}:{s['line']})"
        assert any(_sig_accepts(sig, s["positional_kinds"], s["keyword_kinds"]) for sig in sigs), \
            f"{s['file']}:{s['line']} {s['method']}{tuple(s['positional_kinds'])} matches no glue method {sigs}"


def test_glue_methods_accept_every_device_form_the_extension_accepts():
    """For T = Float64, every device argument form (CuArray, contiguous view, strided view, reshape of a view)
    that a CUDA-extension method accepts in a position, the glue method of the same name accepts too."""
    gold = json.load(open(GOLD))
    glue = glue_methods()
    assert len(gold["ext_methods"]) >= 6
    for e in gold["ext_methods"]:
        sigs = [g for g in glue.get(e["method"], []) if len(g[0]) == len(e["positional"])]
        assert sigs, f"no glue method {e['method']} with {len(e['positional'])} positional parameters"
        pos, _ = sigs[0]
        for (nm, edecl), (gnm, gdecl) in zip(e["positional"], pos):
            # representative element type / rank: the extension's when it states one, else the glue's
            ref = gdecl or edecl or "AnyCuArray{ComplexF64,3}"
            mm = re.fullmatch(r"(?:Union\{Nothing,\s*)?(\w+)(?:\{(.*?)\})?\}?", edecl or ref)
            params = split_top(mm.group(2)) if mm and mm.group(2) else []
            gm = re.fullmatch(r"(?:Union\{Nothing,\s*)?(\w+)(?:\{(.*?)\})?\}?", ref)
            gparams = split_top(gm.group(2)) if gm and gm.group(2) else []
            elt = _norm_elt(params[0]) if params and _norm_elt(params[0]) else (
                _norm_elt(gparams[0]) if gparams else "ComplexF64")
            nd = params[1] if len(params) > 1 else (gparams[1] if len(gparams) > 1 else str(
                ALIAS.get(gm.group(1) if gm else "", (None, None))[1] or 3))
            if edecl in ("Int", "Char"):
                kinds = ["int" if edecl == "Int" else "char"]
            else:
                kinds = [f"dev:{elt}:{nd}", f"view:{elt}:{nd}:dense", f"view:{elt}:{nd}:strided", f"rview:{elt}:{nd}"]
            for k in kinds:
                if accepts(edecl, k):
                    assert accepts(gdecl, k), f"{e['method']} parameter {nm}: extension {edecl} takes {k}, glue {gdecl} does not"
