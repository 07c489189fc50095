"""Outer-q batched loop (host mirror of epb_eph_outer_q).

`run_eph_over_q_and_k` follows the reference's batched outer-q driver
(src/calculator/run_eph_over_q_and_k.jl:428-613): per q, g(Re, q) in the phonon eigenmode (or Cartesian)
basis; per batch of k, the k+q eigensolve, the window masks on both sides and ep = ukq^H g(k, q) uk; each
calculator receives the EPDataKBatched payload (src/EPData.jl:76-114) as torch views of the device
buffers, ordered on the context's stream. Calculators are objects with `run_batch(payload)` and
optionally `begin_q(iq)` / `end_q(iq)` (calculator_begin!/end! of OuterIteration); an exception inside
one aborts the loop with EpbError.

The loop also returns, for every q, the gauge-invariant record A[iq] = sum_k wtk sum |ep|^2 that the
reference's tests accumulate (test/test_gpu.jl:589-654).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import PREC_FP64, check

_DT = {"c128": ("<c16", 16), "f64": ("<f8", 8), "f32": ("<f4", 4), "i32": ("<i4", 4)}


class _DevView:
    """__cuda_array_interface__ over a raw device pointer (Julia column-major shape). torch accepts only
    writable views; the payload is read-only by contract (the loop reuses the buffers next batch)."""

    def __init__(self, ptr, shape, kind, stream):
        typestr, item = _DT[kind]
        jl = tuple(int(n) for n in shape)
        self.__cuda_array_interface__ = {
            "shape": tuple(reversed(jl)), "typestr": typestr, "data": (int(ptr or 0), False), "version": 3,
            "strides": None, "stream": None,
        }


def _view(ptr, shape, kind, stream):
    import torch

    if any(n == 0 for n in shape):
        dt = {"c128": torch.complex128, "f64": torch.float64, "f32": torch.float32, "i32": torch.int32}[kind]
        return torch.empty(tuple(reversed(shape)), dtype=dt, device="cuda")
    return torch.as_tensor(_DevView(ptr, shape, kind, stream), device="cuda")


class KBatch:
    """EPDataKBatched: eps (nw, nw, nm, nk), ek / ekq (nw, nk), uk / ukq (nw, nw, nk), wtk (nk), xks (3, nk),
    ik (nk), omega (nm), iq, k0; tensors in the Julia byte layout (torch shape reversed)."""

    def __init__(self, p):
        nw, nm, nk = p.nw, p.nm, p.nk
        s = p.stream
        self.iq, self.k0, self.nk = p.iq, p.k0, nk
        self.eps = _view(p.eps, (nw, nw, nm, nk), "c128", s) if p.eps else None
        self.ek = _view(p.ek, (nw, nk), "f64", s)
        self.ekq = _view(p.ekq, (nw, nk), "f64", s)
        self.uk = _view(p.uk, (nw, nw, nk), "c128", s)
        self.ukq = _view(p.ukq, (nw, nw, nk), "c128", s)
        self.wtk = _view(p.wtk, (nk,), "f64", s)
        self.xks = _view(p.xk, (3, nk), "f64", s)
        self.ik = _view(p.ik, (nk,), "i32", s)
        self.omega = _view(p.omega, (nm,), "f64", s)


def _wrap(calc, errors):
    def begin(user, iq, stream):
        try:
            if hasattr(calc, "begin_q"):
                calc.begin_q(int(iq))
            return 0
        except BaseException as e:  # reported after the loop returns
            errors.append(e)
            return 1

    def run(user, pp):
        try:
            calc.run_batch(KBatch(pp.contents))
            return 0
        except BaseException as e:
            errors.append(e)
            return 1

    def end(user, iq, stream):
        try:
            if hasattr(calc, "end_q"):
                calc.end_q(int(iq))
            return 0
        except BaseException as e:
            errors.append(e)
            return 1

    fns = (_lib.BEGIN_Q_FN(begin), _lib.RUN_BATCH_FN(run), _lib.END_Q_FN(end))
    return _lib.OuterQCalc(fns[0], fns[1], fns[2], None), fns


def run_eph_over_q_and_k(dm, xks, xqs, *, wtk=None, window_k=(-math.inf, math.inf),
                         window_kq=(-math.inf, math.inf), calculators=(), prec=PREC_FP64,
                         eph_phonon_basis="eigenmode", nk_batch_max=0, q_chunk=0):
    """(A (nq,), stats) for the model `dm` (pipeline.DeviceModel); xks (3, nk), xqs (3, nq) host arrays."""
    if eph_phonon_basis not in ("eigenmode", "cartesian"):
        raise ValueError(f"eph_phonon_basis must be 'eigenmode' or 'cartesian', got {eph_phonon_basis!r}")
    for c in calculators:
        if not hasattr(c, "run_batch"):
            raise TypeError(f"{c!r} has no run_batch(payload): it does not support the EPDataKBatched payload")
    xk = np.ascontiguousarray(np.asarray(xks, dtype=np.float64).reshape(3, -1).T)
    xq = np.ascontiguousarray(np.asarray(xqs, dtype=np.float64).reshape(3, -1).T)
    nk, nq = xk.shape[0], xq.shape[0]
    w = None if wtk is None else np.ascontiguousarray(np.asarray(wtk, dtype=np.float64).reshape(-1))
    if w is not None and w.shape[0] != nk:
        raise ValueError(f"wtk has {w.shape[0]} entries for {nk} k points")
    p = _lib.OuterQParams()
    p.wmin_k, p.wmax_k = float(window_k[0]), float(window_k[1])
    p.wmin_kq, p.wmax_kq = float(window_kq[0]), float(window_kq[1])
    p.k_batch, p.q_chunk, p.prec = int(nk_batch_max), int(q_chunk), int(prec)
    p.phonon_basis = 0 if eph_phonon_basis == "eigenmode" else 1
    errors, keep = [], []
    arr = (_lib.OuterQCalc * max(len(calculators), 1))()
    for i, c in enumerate(calculators):
        arr[i], fns = _wrap(c, errors)
        keep.append(fns)
    A = np.zeros(max(nq, 1))
    stats = (C.c_int64 * 4)()
    st = _lib.lib().epb_eph_outer_q(dm.ctx.h, dm.h, xk.ctypes.data if nk else None,
                                    w.ctypes.data if w is not None and nk else None, nk,
                                    xq.ctypes.data if nq else None, nq, C.byref(p), arr, len(calculators),
                                    A.ctypes.data, stats)
    if errors:
        raise errors[0]
    check(st)
    return A[:nq], dict(kept_k=stats[0], k_batch=stats[1], q_chunk=stats[2], batches=stats[3])
