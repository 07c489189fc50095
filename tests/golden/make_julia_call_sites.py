"""Extract the reference's device call sites of the methods the Julia glue overrides (fixture generator).

Reads the reference sources (default /root/reference, or the path given) and writes
julia_call_sites.json beside this script: for every call of an overridden method on the GPU path, the
file:line, the argument texts (positional and keyword) and each argument's kind, derived from a table of
the identifiers at those sites whose construction line is checked against the source here. Kinds:
  dev:<eltype>:<ndims>           a device array (CuArray: alloc / similar / CuArray / a reshape of one)
  view:<eltype>:<ndims>:dense    a contiguous view of a device array (FastContiguousSubArray)
  view:<eltype>:<ndims>:strided  any other view
  rview:<eltype>:<ndims>         a reshape of a view (ReshapedArray wrapping a SubArray)
  host-kvec / itp / char / int / range / nothing / any
Run: python tests/golden/make_julia_call_sites.py [/path/to/reference]
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "julia_call_sites.json")

# Methods the glue overrides, and the reference files whose GPU-path calls of them are checked.
METHODS = ["fourier_phase!", "get_fourier_batched!", "eigvals_batched", "eigen_batched", "batched_gemm!",
           "get_eph_RR_to_kR_batched!", "get_eph_kR_to_kq_batched!", "eph_apply_rotations!",
           "get_eph_Rq_to_kq_batched!", "eph_window_scatter!", "bte_window_accumulate!"]
FILES = ["src/calculator/run_eph_over_k_and_kq.jl", "src/calculator/run_eph_over_q_and_k.jl",
         "src/wannier/batched_fourier_core.jl", "src/wannier_to_bloch_batched.jl",
         "src/boltzmann/boltzmann_calculator.jl"]

# identifier -> (kind, a construction text that must occur in the file of the call)
C, F, I = "ComplexF64", "Float64", "Int"
IDENT = {
    # run_eph_over_k_and_kq.jl (backend = gpu_backend(): `alloc` makes CuArrays)
    "P_mk": (f"dev:{C}:2", "P_mk  = alloc(backend, Complex{FT}, nr_ep, nk_batch_max)"),
    "P_kq": (f"dev:{C}:2", "P_kq = alloc(backend, Complex{FT}, nr_ep, nq_batch_max)"),
    "irvecp_mat": (f"dev:{F}:2", "irvecp_mat = _irvec_to_device_matrix(model.epmat.irvec_next, epmat_dev, FT)"),
    "mxk_dev": (f"dev:{F}:2", "mxk_dev = _kpoints_to_device_matrix(backend, kpts) .* -1"),
    "xkq_dev": (f"dev:{F}:2", "xkq_dev = _kpoints_to_device_matrix(backend, kqpts)"),
    "ep_ekpR_all": (f"dev:{C}:3", "ep_ekpR_all = alloc(backend"),
    "uks_dev": (f"dev:{C}:3", "uks_dev"),
    "epkq_dev": (f"dev:{C}:4", "epkq_dev"),
    "uphs_dev": (f"dev:{C}:3", "uphs_dev"),
    "ukqs_all_dev": (f"dev:{C}:3", "ukqs_all_dev"),
    "g2_dev": (f"dev:{F}:4", "g2_dev    = alloc(backend, FT, nw, nbandk_max, nmodes, nq_batch_max)"),
    "ωq_dev": (f"dev:{F}:2", "ωq_dev    = alloc(backend, FT, nmodes, nq_batch_max)"),
    "ukqs_used": (f"view:{C}:3:dense", "ukqs_used = view(ukqs_all_dev, :, :, qstart:qend)"),
    "itp_epmat": ("itp", "itp_epmat"),
    "ks_batch": ("host-kvec", "ks_batch"),
    "kRkq_ws": ("any", "kRkq_ws"),
    # run_eph_over_q_and_k.jl
    "Hkq_flat": (f"dev:{C}:2", "Hkq_flat"),
    "itp_el_ham": ("itp", "itp_el_ham"),
    "kqs_batch": ("host-kvec", "kqs_batch"),
    "ep_batch": (f"dev:{C}:4", "ep_batch"),
    "itp_ep_eRpq": ("itp", "itp_ep_eRpq"),
    "Uk_batch": (f"dev:{C}:3", "Uk_batch"),
    "Ukq_batch": (f"dev:{C}:3", "Ukq_batch"),
    "ep_ws": ("any", "ep_ws"),
    # batched_fourier_core.jl (core buffers on the device of parent.op_r)
    "phase": (f"dev:{C}:2", "phase"),
    "irvec_mat": (f"dev:{F}:2", "irvec_mat = _irvec_to_device_matrix(parent.irvec, parent, T)"),
    "xkmat": (f"dev:{F}:2", "xkmat"),
    # wannier_to_bloch_batched.jl (generic drivers still reached on the device)
    "Hk": (f"dev:{C}:2", "Hk = similar(ham.op_r, Complex{T}, ham.ndata, nk)"),
    "Vk": (f"dev:{C}:2", "Vk = similar(vel.op_r, Complex{T}, vel.ndata, nk)"),
    "Vb": (f"dev:{C}:3", "Vb = reshape(Vk, nw, nw, 3 * nk)"),
    "ub": (f"dev:{C}:3", "ub = reshape(urep, nw, nw, 3 * nk)"),
    "tmp": (f"dev:{C}:3", "tmp = similar(Vb)"),
    "out": (f"dev:{C}:3", "out = similar(Vb)"),
    "ukqs": (f"dev:{C}:3", "ukqs"),
    "uks": (f"dev:{C}:3", "uks"),
    "mmats": (f"dev:{C}:3", "mmats"),
    "itp": ("itp", "itp"),
    "xk_list": ("host-kvec", "xk_list"),
    # boltzmann_calculator.jl (device buffers of the calculator's setup; tile arrays)
    "g2s": (f"view:{F}:4:dense", "g2s"),
    "ωqs": (f"view:{F}:2:dense", "ωqs"),
    "imap_i_at_k": (f"view:{I}:1:dense", "imap_i_at_k = view(dev.imap_i, ibandk_offset+1:ibandk_offset+nbandk, ik)"),
    "ikqs": ("range", "ikqs"),
    "dev.Sₒ": (f"dev:{F}:2", "fill!(alloc(backend, FT, n_i, nT), zero(FT)),                       # Sₒ"),
    "device_array(t, 1)": (f"dev:{F}:3", "device_array(t, 1)"),
    "dev.imap_f": (f"dev:{I}:2", "_indmap_to_device(backend, calc.el_f, calc.nw),                     # imap_f"),
    "dev.e_i": (f"dev:{F}:1", "to_device(backend, calc.el_i.es),"),
    "dev.e_f": (f"dev:{F}:1", "to_device(backend, calc.el_f.es),"),
    "dev.wf": (f"dev:{F}:1", "to_device(backend, collect(FT, state_weights(calc.el_f))),"),
    "dev.μ": (f"dev:{F}:1", "to_device(backend, collect(FT, calc.occ.μlist)),"),
    "dev.T": (f"dev:{F}:1", "to_device(backend, collect(FT, calc.occ.Tlist)),"),
    "dev.smearing": (f"dev:{F}:1", "to_device(backend, calc.smearing_list),"),
    "calc.occupation_method": ("int", "calc.occupation_method"),
    "calc.omega_cutoff": ("any", "calc.omega_cutoff"),
    "tile_offset(t)": ("int", "tile_offset(t)"),
}
# Names whose value is an integer index or a range in the index position of a view.
SCALARS = {"ik_ind", "ik", "nk", "nk_batch", "qstart", "qend", "nq_batch", "nw", "nk_batch_max", "nbandk",
           "nbandkq", "nmodes", "i0", "method"}
# (file, enclosing function): generic methods the glue replaces wholesale; calls inside them are not
# reached on the device path
UNREACHED = {("src/wannier_to_bloch_batched.jl", f) for f in (
    "get_eph_RR_to_kR_batched!", "get_eph_kR_to_kq_batched!", "get_eph_Rq_to_kq_batched!", "eph_apply_rotations!",
    "eph_apply_rotations_rqkq!")}
RANGES = {"rng_q", "iks_batch", "rng_k"}


def split_top(s):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch in ",;" and depth == 0:
            out.append((cur.strip(), ch))
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append((cur.strip(), ""))
    return out


def index_kind(ix):
    ix = ix.strip()
    if ix == ":":
        return "colon"
    if ix in RANGES or re.fullmatch(r"[\w+\-*]+\s*:\s*[\w+\-*]+", ix):
        return "range"
    if ix in SCALARS or re.fullmatch(r"\d+", ix):
        return "int"
    raise KeyError(f"unknown index expression {ix!r}")


def view_kind(base, indices):
    k = classify(base)
    assert k.startswith("dev:"), (base, k)
    _, et, _nd = k.split(":")
    kinds = [index_kind(i) for i in indices]
    nd = sum(x != "int" for x in kinds)
    # FastContiguousSubArray: colons, then at most one range, then only integer indices
    seen_range, dense = False, True
    for x in kinds:
        if x == "colon" and not seen_range:
            continue
        if x == "range" and not seen_range:
            seen_range = True
            continue
        if x == "int":
            seen_range = True
            continue
        dense = False
    return f"view:{et}:{nd}:{'dense' if dense else 'strided'}"


def classify(expr):
    e = expr.strip()
    if e.startswith("@views "):
        e = e[len("@views "):].strip()
    if "=" in e and not e.startswith(("view(", "reshape(")) and re.match(r"^[\wωₒᵢ]+\s*=", e):
        e = e.split("=", 1)[1].strip()           # keyword argument
    if e in ("'N'", "'T'", "'C'"):
        return "char"
    if e == "nothing":
        return "nothing"
    m = re.fullmatch(r"view\((.*)\)", e, flags=re.S)
    if m:
        parts = [p for p, _ in split_top(m.group(1))]
        return view_kind(parts[0], parts[1:])
    m = re.fullmatch(r"([\wωₒᵢ]+)\[(.*)\]", e, flags=re.S)  # inside @views
    if m:
        return view_kind(m.group(1), [p for p, _ in split_top(m.group(2))])
    m = re.fullmatch(r"reshape\((.*)\)", e, flags=re.S)
    if m:
        parts = [p for p, _ in split_top(m.group(1))]
        inner = classify(parts[0])
        et = inner.split(":")[1]
        nd = len(parts) - 1
        return f"dev:{et}:{nd}" if inner.startswith("dev:") else f"rview:{et}:{nd}"
    m = re.fullmatch(r"_fourier_hk_batched\(.*\)", e)
    if m:
        return f"dev:{C}:3"  # reshape(Hk, nw, nw, nk) of a similar() buffer
    if e in IDENT:
        return IDENT[e][0]
    if e in SCALARS:
        return "int"
    raise KeyError(f"unclassified argument {expr!r}")


def calls_in(path, rel):
    txt = open(path).read()
    lines = txt.split("\n")
    in_doc, state = [], False  # lines inside a triple-quoted docstring
    for ln in lines:
        n = ln.count('"""')
        in_doc.append(state or n > 0)
        if n % 2:
            state = not state
    found = []
    for name in METHODS:
        for m in re.finditer(r"(?<![\w.])" + re.escape(name) + r"\(", txt):
            line_no = txt.count("\n", 0, m.start()) + 1
            line = lines[line_no - 1]
            stripped = line.strip()
            if stripped.startswith(("#", "function ")) or "`" in line[: m.start() - txt.rfind("\n", 0, m.start())]:
                continue
            if in_doc[line_no - 1]:
                continue
            i, depth = m.end() - 1, 0
            for j in range(i, len(txt)):
                depth += txt[j] == "("
                depth -= txt[j] == ")"
                if depth == 0:
                    break
            body = txt[i + 1:j]
            prefix = line[: len(line) - len(line.lstrip())]
            at_views = stripped.startswith("@views")
            parts = split_top(" ".join(body.split()))
            pos, kw, in_kw = [], [], False
            for p, sep in parts:
                (kw if in_kw else pos).append(p)
                if sep == ";":
                    in_kw = True
            encl = None
            for j in range(line_no - 1, -1, -1):
                fm = re.match(r"^function\s+([\w!]+)\(", lines[j])
                if fm:
                    encl = fm.group(1)
                    break
                if lines[j].startswith("end"):
                    break
            if (rel, encl) in UNREACHED:
                continue
            found.append({"file": rel, "line": line_no, "method": name, "views_macro": at_views,
                          "positional": pos, "keywords": kw})
    return found


def build(ref):
    sites = []
    for rel in FILES:
        sites += calls_in(os.path.join(ref, rel), rel)
    for s in sites:
        src = open(os.path.join(ref, s["file"])).read()
        pre = "@views " if s["views_macro"] else ""
        s["positional_kinds"] = [classify(pre + a if pre and "[" in a else a) for a in s["positional"]]
        s["keyword_kinds"] = {a.split("=", 1)[0].strip(): classify(a) for a in s["keywords"] if "=" in a}
        for a in s["positional"] + [k.split("=", 1)[-1] for k in s["keywords"]]:
            base = re.split(r"[\[(,]", a.strip().replace("view(", "").replace("reshape(", ""))[0].strip()
            if base in IDENT:
                assert IDENT[base][1] in src, f"{s['file']}: construction of {base} not found: {IDENT[base][1]!r}"
    sites.sort(key=lambda s: (s["file"], s["line"]))
    return sites


def ext_methods(ref):
    """The CUDA extension's methods of the overridden names: [{method, line, positional, keywords}] with the
    declared type text of each parameter (None when untyped) and its `where` clause."""
    rel = "ext/ElectronPhononCUDAExt.jl"
    txt = open(os.path.join(ref, rel)).read()
    out = []
    for m in re.finditer(r"^function ElectronPhonon\.([\w!]+)\(", txt, flags=re.M):
        name = m.group(1)
        if name not in METHODS:
            continue
        i, depth = m.end() - 1, 0
        for j in range(i, len(txt)):
            depth += txt[j] == "("
            depth -= txt[j] == ")"
            if depth == 0:
                break
        rest = txt[j + 1: txt.index("\n", j)]
        where = re.search(r"where\s*\{?([^}]*)\}?", rest)
        pos, kw, in_kw = [], [], False
        for p, sep in split_top(" ".join(txt[i + 1:j].split())):
            nm, _, ty = p.split("=", 1)[0].strip().partition("::")
            (kw if in_kw else pos).append([nm.strip(), ty.strip() or None])
            if sep == ";":
                in_kw = True
        out.append({"method": name, "line": txt.count("\n", 0, m.start()) + 1, "positional": pos, "keywords": kw,
                    "where": where.group(1).strip() if where else None})
    return out


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    sites = build(ref)
    ext = ext_methods(ref)
    with open(OUT, "w") as fh:
        json.dump({"reference": "jaemolihm/ElectronPhonon.jl", "sites": sites, "ext_methods": ext}, fh, indent=1,
                  ensure_ascii=False)
    print(f"{len(sites)} call sites, {len(ext)} extension methods -> {OUT}")
