"""The ctypes mirrors of the C-ABI structs match include/epb200.h field for field (no GPU).

A C probe compiled with gcc against the header prints sizeof and every field's offsetof; each ctypes
Structure of epb200/_lib.py must report the same size, field names and offsets, so no argument struct
crosses the boundary misaligned.
"""
import ctypes
import os
import shutil
import subprocess

import pytest

from epb200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PAIRS = [("epb_window_stats", _lib.WindowStats), ("epb_bte_params", _lib.BteParams),
         ("epb_tiled_info", _lib.TiledInfo), ("epb_outer_q_params", _lib.OuterQParams),
         ("epb_kbatch_payload", _lib.KBatchPayload), ("epb_outer_q_calc", _lib.OuterQCalc),
         ("epb_mlp_train_opts", _lib.MlpTrainOpts)]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "epb200.h"', 'int main(void) {']
    for cname, cls in PAIRS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            cname, field, val = line.split()
            got[(cname, field)] = int(val)
    for cname, cls in PAIRS:
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])
