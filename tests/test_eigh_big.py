"""Eigensolver orders 65..96 and uneven (varlen) batches vs LAPACK ZHEEV (the config-3 shape).

Tolerances: eigenvalues within 1e-11 (mixed: FP32 Jacobi + FP64 refinement) / 1e-12 (FP64 mode)
of the largest |eigenvalue|; U diag(E) U^H reconstructs H within 10x that; U^H U = I within 1e-11 n.
Planted clusters (2-4 eigenvalues spaced 1e-10): eigenvalues as above and the cluster projector
sum_{i in c} u_i u_i^H within 1e-8 of LAPACK's (individual vectors inside a cluster are only
defined to ~1e-14 / 1e-10).
"""
import numpy as np
import pytest

from oracle import epb_oracle as O
from epb200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def B(gpu_lib):
    from epb200 import batched

    return batched


def _check(es, us, mats, tol):
    for e, u, h in zip(es, us, mats):
        n = h.shape[0]
        eref, uref = O._zheev(h.copy(), "V")
        scale = max(np.abs(eref).max(), 1.0)
        assert np.max(np.abs(e - eref)) <= tol * scale, (n, np.max(np.abs(e - eref)))
        rec = u @ np.diag(e) @ u.conj().T
        hf = np.triu(h) + np.triu(h, 1).conj().T
        np.fill_diagonal(hf, np.real(np.diag(h)))
        assert np.max(np.abs(rec - hf)) <= 10 * tol * scale, n
        assert np.max(np.abs(u.conj().T @ u - np.eye(n))) <= 1e-11 * n, n
        # clusters of the reference spectrum: projectors agree
        gaps = np.diff(eref)
        start = 0
        for i in range(1, n + 1):
            if i == n or gaps[i - 1] > 1e-6 * scale:
                if i - start > 1:
                    p = u[:, start:i] @ u[:, start:i].conj().T
                    pr = uref[:, start:i] @ uref[:, start:i].conj().T
                    assert np.max(np.abs(p - pr)) <= 1e-8, (n, start, i)
                start = i


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n", [65, 72, 96])
def test_eigh_uniform_large(B, n, prec):
    rng = np.random.default_rng(n + 100 * prec)
    nk = 21
    a = rng.standard_normal((n, n, nk)) + 1j * rng.standard_normal((n, n, nk))
    h = np.asfortranarray((a + a.conj().transpose(1, 0, 2)) / 2)
    E, U = B.eigen_batched(B.jl(h), prec=prec)
    E, U = B.host(E), B.host(U)
    tol = 1e-12 if prec == 0 else 1e-11
    _check([E[:, k] for k in range(nk)], [U[:, :, k] for k in range(nk)], [h[:, :, k] for k in range(nk)], tol)


@pytest.mark.parametrize("prec", [0, 1])
def test_eigh_varlen_config3_shape(B, prec):
    """Orders 4..96, a quarter with planted 2-4-fold clusters spaced 1e-10."""
    ns, mats = synth.config3_matrices(240, seed=17 + prec, degenerate_frac=0.25)
    es, us = B.eigen_varlen(mats, prec=prec)
    tol = 1e-12 if prec == 0 else 1e-11
    _check(es, us, mats, 10 * tol)


def test_eigh_varlen_bad_order_reported(B):
    from epb200._lib import EpbError

    rng = np.random.default_rng(5)
    mats = []
    for n in (5, 100, 70):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        mats.append(np.asfortranarray((a + a.conj().T) / 2))
    with pytest.raises(EpbError):
        B.eigen_varlen(mats)
    # the supported orders are still solved
    vb = B.VarlenBatch(mats)
    from epb200 import _lib

    st = _lib.lib().epb_eigh_varlen(B._ctx().h, B.ptr(vb.A), B.ptr(vb.a_off), B.ptr(vb.n), 3, B.ptr(vb.E),
                                    B.ptr(vb.e_off), b"V", 0)
    assert st == _lib.EPB_ERR_ARG
    es, _ = vb.unpack()
    for k in (0, 2):
        np.testing.assert_allclose(es[k], O._zheev(mats[k].copy(), "N")[0], atol=1e-11 * np.abs(es[k]).max())


@pytest.mark.parametrize("prec", [0, 1])
def test_eigh_varlen_async_graph_capture(B, prec):
    """The read-back-free varlen solve (epb_eigh_varlen_async) captured in a CUDA graph after one eager call
    sized the workspace: a replay on the refilled batch equals the eager solve bit for bit and matches
    LAPACK; epb_eigh_status reports an order outside 1..96 that a replayed batch contains."""
    import torch

    from epb200 import _lib

    L = _lib.lib()
    s = torch.cuda.Stream()
    ctx = _lib.Context(0, s)
    for bad in (False, True):
        ns, mats = synth.config3_matrices(48, seed=31 + prec, degenerate_frac=0.25)
        if bad:
            rng = np.random.default_rng(3)
            a = rng.standard_normal((100, 100)) + 1j * rng.standard_normal((100, 100))
            mats = mats[:20] + [np.asfortranarray((a + a.conj().T) / 2)] + mats[20:]
        vb = B.VarlenBatch(mats)
        A0 = vb.A.clone()
        args = (ctx.h, B.ptr(vb.A), B.ptr(vb.a_off), B.ptr(vb.n), len(mats), B.ptr(vb.E), B.ptr(vb.e_off), b"V", prec)
        vb.E.zero_()  # the slots of a skipped (unsupported) matrix are left as they were
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            _lib.check(L.epb_eigh_varlen_async(*args))
        st = L.epb_eigh_status(ctx.h)
        assert st == (_lib.EPB_ERR_ARG if bad else _lib.EPB_OK)
        E_eager, A_eager = vb.E.clone(), vb.A.clone()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            _lib.check(L.epb_eigh_varlen_async(*args))
        vb.A.copy_(A0)
        vb.E.zero_()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        st = L.epb_eigh_status(ctx.h)
        assert st == (_lib.EPB_ERR_ARG if bad else _lib.EPB_OK)
        assert torch.equal(vb.E, E_eager) and torch.equal(vb.A, A_eager)
        es, us = vb.unpack()
        keep = [i for i, m in enumerate(mats) if m.shape[0] <= 96]
        _check([es[i] for i in keep], [us[i] for i in keep], [mats[i] for i in keep], 1e-11 if prec == 0 else 1e-10)
        del g


def test_eigh_varlen_autotuned_classes(B):
    """The mixed varlen call times both candidate kernels of the classes 17..32, 33..48, 49..64 and 65..80
    on its first batch (on a copy of the batch) and keeps the faster in the context's tuning table; each
    candidate is accurate, and a second context given the table's text solves bit for bit alike without
    timing."""
    import torch

    from epb200 import _lib

    L = _lib.lib()
    ns, mats = synth.config3_matrices(160, seed=41, degenerate_frac=0.25)
    keys = ["eigh_varlen/16/32/1", "eigh_varlen/32/48/1", "eigh_varlen/48/64/1", "eigh_varlen/64/80/1"]
    outs = []
    for forced in (None, 0, 1):
        s = torch.cuda.Stream()
        ctx = _lib.Context(0, s)
        if forced is not None:  # every class on the given candidate
            t = _lib.TuneTable("".join(f"{k} {forced}\n" for k in keys))
            t.import_into(ctx)
        vb = B.VarlenBatch(mats)
        with torch.cuda.stream(s):
            _lib.check(L.epb_eigh_varlen(ctx.h, B.ptr(vb.A), B.ptr(vb.a_off), B.ptr(vb.n), len(mats), B.ptr(vb.E),
                                         B.ptr(vb.e_off), b"V", 1))
        torch.cuda.synchronize()
        table = _lib.TuneTable(ctx.tune_text())
        assert all(table.get(k) in (0, 1) for k in keys), ctx.tune_text()
        es, us = vb.unpack()
        _check(es, us, mats, 1e-10)
        outs.append((table, vb.E.clone(), vb.A.clone()))
    # replay of the autotuned choices from the table text
    s = torch.cuda.Stream()
    ctx = _lib.Context(0, s)
    outs[0][0].import_into(ctx)
    vb = B.VarlenBatch(mats)
    with torch.cuda.stream(s):
        _lib.check(L.epb_eigh_varlen(ctx.h, B.ptr(vb.A), B.ptr(vb.a_off), B.ptr(vb.n), len(mats), B.ptr(vb.E),
                                     B.ptr(vb.e_off), b"V", 1))
    torch.cuda.synchronize()
    assert torch.equal(vb.E, outs[0][1]) and torch.equal(vb.A, outs[0][2])
