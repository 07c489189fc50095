"""Whole e-ph pass driver over the C ABI (epb_model_create / epb_eph_pass).

`run_eph_over_k_and_q` mirrors the reference driver of the same name
(src/calculator/run_eph_over_k_and_q.jl:17,230-340: arbitrary k x arbitrary q, q convention), run
the batched way of the GPU outer-k loop (src/calculator/run_eph_over_k_and_kq.jl:792-892). Its
built-in consumer reduces g2 in place to `g2sum[nu, k]` and keeps the full g2 block of every
`sample_stride`-th q, because a full pass produces ~5e10 values.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import PREC_FP64, PREC_MIXED, check, ptr  # noqa: F401
from .batched import jl, jl_empty


@dataclass
class PassResult:
    ek: object        # (nw, nk) device float64
    omega: object     # (nm, nq)
    g2sum: object     # (nm, nk)
    g2_sample: object  # (nw, nw, nm, nsamp, nk) or None
    n_elements: int
    sample_stride: int
    k_batch: int = 0  # inner k batch the library used (autotuned when not given)
    rot_variant: int = -1  # rotation kernel of the mixed pass (0 warp tensor cores, 1 FP32; -1 FP64 pass)
    kq_form: int = -1      # kR->kq GEMM form of the mixed pass (1 A-resident, 0 streamed; -1 FP64 pass)


class DeviceModel:
    """Device copy of a model's hot-path operators plus the library's epb_model handle.

    Mirrors `to_device(::GPUBackend, model)` usage in the reference GPU loop
    (src/calculator/run_eph_over_k_and_kq.jl:271): the operators are uploaded once, outside any
    timed region; `mixed=True` also prepares the split-BF16 operand planes.
    """

    def __init__(self, model, mixed=False, device="cuda", ctx=None):
        import torch

        self.nw, self.nm = model.nw, model.nmodes
        self.ham = jl(model.el_ham.op_r, device)
        self.dyn = jl(model.ph_dyn.op_r, device)
        self.mass = torch.as_tensor(np.asarray(model.mass, dtype=np.float64), device=device)
        ep = model.epmat.op_r
        self.epmat = ep if isinstance(ep, torch.Tensor) else jl(ep, device)
        self.irvec_el = np.ascontiguousarray(model.el_ham.irvec, dtype=np.int64)
        self.irvec_ph = np.ascontiguousarray(model.ph_dyn.irvec, dtype=np.int64)
        self.irvec_ep = np.ascontiguousarray(model.epmat.irvec_next, dtype=np.int64)
        assert np.array_equal(model.epmat.irvec, model.el_ham.irvec), "epmat Re grid must equal the H grid"
        self.ctx = ctx if ctx is not None else _lib.default_context()
        h = C.c_void_p()
        check(_lib.lib().epb_model_create(
            self.ctx.h, ptr(self.ham), self.nw, self.irvec_el.ctypes.data, self.irvec_el.shape[0],
            ptr(self.dyn), ptr(self.mass), self.nm, self.irvec_ph.ctypes.data, self.irvec_ph.shape[0],
            ptr(self.epmat), self.irvec_ep.ctypes.data, self.irvec_ep.shape[0], 1 if mixed else 0, C.byref(h)))
        self.h = h
        self.mixed = mixed

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().epb_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_eph_over_k_and_q(dm: DeviceModel, xks, xqs, *, prec=PREC_FP64, k_batch=16, sample_stride=None,
                         out=None):
    """Full-band pass over the k list `xks` (3, nk) and the q list `xqs` (3, nq) (device float64 tensors
    in Julia layout, or numpy arrays). Returns a PassResult with device tensors. k_batch <= 0 (or None)
    lets the library's autotuner choose the inner k batch (`PassResult.k_batch` reports it)."""
    import torch

    xk = xks if isinstance(xks, torch.Tensor) else jl(np.asfortranarray(xks, dtype=np.float64))
    xq = xqs if isinstance(xqs, torch.Tensor) else jl(np.asfortranarray(xqs, dtype=np.float64))
    nk, nq = xk.numel() // 3, xq.numel() // 3
    nw, nm = dm.nw, dm.nm
    if out is None:
        nsamp = 0 if sample_stride is None else -(-nq // sample_stride)
        out = PassResult(
            ek=jl_empty((nw, nk), torch.float64), omega=jl_empty((nm, nq), torch.float64),
            g2sum=jl_empty((nm, nk), torch.float64),
            g2_sample=None if sample_stride is None else jl_empty((nw, nw, nm, nsamp, nk), torch.float64),
            n_elements=0, sample_stride=sample_stride or 0)
    stats = np.zeros(4, dtype=np.int64)
    check(_lib.lib().epb_eph_pass(dm.ctx.h, dm.h, ptr(xk), nk, ptr(xq), nq, int(prec), int(k_batch or 0),
                                  int(sample_stride or 1), ptr(out.ek), ptr(out.omega), ptr(out.g2sum),
                                  ptr(out.g2_sample), stats.ctypes.data))
    out.n_elements = int(stats[0])
    out.k_batch = int(stats[1])
    out.rot_variant = int(stats[2])
    out.kq_form = int(stats[3])
    return out
