"""CPU restatement of the reference's `read_epmat` (src/model_new.jl:487-568) (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only `tests/` may import it. It reads the raw
`<prefix>.epmatwp` (complex128, EPW order (iw, jw, iRe, imode, iRp)), applies the R sort, the
Wigner-Seitz divisions in the reference's order and the "el" / "ph" layout with numpy. Parity unpinned
against the reference's own files: the EPW artifacts of its tests (test/Artifacts.toml) are not present;
the restatement is pinned by a round trip through a writer of the same format in tests/test_epw.py.
"""
from __future__ import annotations

import numpy as np


def _div(z, d):
    """z / d for an integer d as Julia's Complex / Real: both parts divided (numpy's complex division
    multiplies by a reciprocal and is not bit-identical)."""
    out = np.empty_like(z)
    out.real = z.real / d
    out.imag = z.imag / d
    return out


def read_epmat(filename, nw, nmodes, nr_el, nr_ep, ind_el, ind_ep, ndegen_el, ndegen_ep, layout="el",
               skip_ndegen_ep=False, ndegen_pre_divided=False):
    """ind_el / ind_ep: 0-based sort permutations (new <- old); ndegen_* already in sorted order."""
    raw = np.fromfile(filename, dtype=np.complex128, count=nw * nw * nr_el * nmodes * nr_ep)
    ep = raw.reshape(nw, nw, nr_el, nmodes, nr_ep, order="F")
    ep = ep[:, :, ind_el, :, :][:, :, :, :, ind_ep]
    if not (skip_ndegen_ep or ndegen_pre_divided):
        if ndegen_ep.shape[0] == 1:
            for ir in range(nr_ep):
                d = ndegen_ep[0, 0, ir]
                ep[..., ir] = 0 if d == 0 else _div(ep[..., ir], d)
        else:
            for ir in range(nr_ep):
                for im in range(nmodes):
                    for iw in range(nw):
                        d = ndegen_ep[iw, im // 3, ir]
                        ep[iw, :, :, im, ir] = 0 if d == 0 else _div(ep[iw, :, :, im, ir], d)
    if not ndegen_pre_divided:
        if ndegen_el.shape[0] == 1:
            for ir in range(nr_el):
                d = ndegen_el[0, 0, ir]
                ep[:, :, ir] = 0 if d == 0 else _div(ep[:, :, ir], d)
        else:
            for ir in range(nr_el):
                for jw in range(nw):
                    for iw in range(nw):
                        d = ndegen_el[iw, jw, ir]
                        ep[iw, jw, ir] = 0 if d == 0 else _div(ep[iw, jw, ir], d)
    if layout == "ph":
        return np.asfortranarray(ep.transpose(0, 1, 3, 2, 4).reshape(nw * nw * nmodes * nr_el, nr_ep, order="F"))
    return np.asfortranarray(ep.transpose(0, 1, 3, 4, 2).reshape(nw * nw * nmodes * nr_ep, nr_el, order="F"))
