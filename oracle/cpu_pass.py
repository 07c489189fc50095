"""Batched CPU e-ph pass (TEST INFRASTRUCTURE / CPU BASELINE ONLY; see epb_oracle.py header).

The reference's batched loop run on its CPU backend (the "validation configuration",
src/calculator/run_eph_over_k_and_kq.jl:584-895 on CPUBackend; README_GPU.md:180-186): one ZGEMM
per Fourier stage (src/wannier/batched_fourier_core.jl:117-139), a per-matrix LAPACK ZHEEV loop
(src/wannier_to_bloch_batched.jl:30-65, src/common/AllocatedLAPACK.jl:82-102), and the two-GEMM
rotations plus the |g|^2/(2 omega) fold (src/wannier_to_bloch_batched.jl:442-455), in the q
convention of run_eph_over_k_and_q (src/calculator/run_eph_over_k_and_q.jl:251-330).

It produces exactly what epb_eph_pass produces (ek, omega, g2sum[nu, k], sampled g2 blocks), so it
serves as the size-scaled parity reference of the GPU pass and as the timed CPU baseline.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack

from .epb_oracle import fourier_batched, fourier_phase


def _zheev_stack(h, want_v=True):
    """ZHEEV ('V'/'N', 'U') over a (n, n, b) stack; returns (E (n, b), U (n, n, b))."""
    n, _, b = h.shape
    e = np.empty((n, b))
    u = np.empty_like(h) if want_v else None
    for i in range(b):
        w, v, info = lapack.zheev(h[:, :, i], compute_v=1 if want_v else 0, lower=0)
        if info != 0:
            raise RuntimeError(f"zheev info={info}")
        e[:, i] = w
        if want_v:
            u[:, :, i] = v
    return e, u


def eph_pass_cpu(model, xks, xqs, sample_stride=None):
    nw, nm = model.nw, model.nmodes
    ham, dyn, ep = model.el_ham, model.ph_dyn, model.epmat
    nr_ep = ep.irvec_next.shape[0]
    nk, nq = xks.shape[1], xqs.shape[1]
    # q side
    dq = fourier_batched(dyn.op_r, nm * nm, dyn.irvec, xqs).reshape(nm, nm, nq, order="F")
    sm = np.sqrt(np.asarray(model.mass))
    dq = dq / sm[:, None, None] / sm[None, :, None]
    lam, uph = _zheev_stack(dq)
    omega = np.where(lam >= 0, np.sqrt(np.abs(lam)), -np.sqrt(np.abs(lam)))
    uph = uph / sm[:, None, None]
    phase = fourier_phase(ep.irvec_next, xqs)                        # (nr_ep, nq)
    # k side
    hk = fourier_batched(ham.op_r, nw * nw, ham.irvec, xks).reshape(nw, nw, nk, order="F")
    ek, uk = _zheev_stack(hk)
    nsamp = 0 if sample_stride is None else -(-nq // sample_stride)
    g2sum = np.zeros((nm, nk))
    samples = None if sample_stride is None else np.zeros((nw, nw, nm, nsamp, nk))
    inv2w = 1.0 / (2.0 * omega)
    for k in range(nk):
        # RR -> kR for this k, rotated on the k leg by uk
        gk = fourier_batched(ep.op_r, ep.op_r.shape[0], ep.irvec, xks[:, k:k + 1])[:, 0]
        gk = gk.reshape(nw, nw, nm * nr_ep, order="F")
        kR = np.einsum("ijm,jn->inm", gk, uk[:, :, k]).reshape(nw * nw * nm, nr_ep, order="F")
        # electrons at k+q
        hkq = fourier_batched(ham.op_r, nw * nw, ham.irvec, xks[:, k:k + 1] + xqs).reshape(nw, nw, nq, order="F")
        _, ukq = _zheev_stack(hkq)
        # kR -> kq and the two rotations
        g = (kR @ phase).reshape(nw, nw, nm, nq, order="F")
        t = np.einsum("imq,inaq->mnaq", ukq.conj(), g)
        epq = np.einsum("mnaq,abq->mnbq", t, uph)
        g2 = np.abs(epq) ** 2 * inv2w[None, None, :, :]
        g2sum[:, k] = g2.sum(axis=(0, 1, 3))
        if samples is not None:
            samples[:, :, :, :, k] = g2[:, :, :, ::sample_stride]
    return dict(ek=ek, omega=omega, g2sum=g2sum, g2_sample=samples, n_elements=nk * nq * nw * nw * nm)
