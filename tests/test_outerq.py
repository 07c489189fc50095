"""Outer-q loop: "el" -> "ph" layout, RR -> Rq (Fourier over Rp + mode rotation), Rq -> kq (Fourier over
Re at a k list + ukq^H g uk), through the C ABI against the FP64 oracle.

Pinning: the reference checks that both loop orders give the same ep (test/test_epmat.jl:45-80,
`≈` i.e. rtol sqrt(eps)) and that the batched Rq -> kq matches the per-k form slice by slice
(test/test_gpu.jl:92-107, rtol 1e-9 on the GPU). The oracle's two orders are compared here at 1e-12.
"""
import numpy as np
import pytest

from oracle import epb_oracle as O
from epb200 import synth


def _model(seed=11, nw=4, natom=2):
    return synth.config2_model(seed=seed, n_el=2, n_ph=1, nw=nw, natom=natom)


def _outer_k(m, xk, xq, uk, ukq, uph):
    ep = m.epmat
    kR = O.get_eph_RR_to_kR(ep.op_r, ep.irvec, ep.irvec_next.shape[0], m.nw, m.nmodes, xk, uk)
    return O.get_eph_kR_to_kq(kR, ep.irvec_next, xq, uph, ukq, uk.shape[1])


def test_oracle_el_to_ph_layout():
    rng = np.random.default_rng(0)
    nw, nm, nr_el, nr_ep = 2, 3, 5, 4
    el = rng.standard_normal((nw, nw, nm, nr_ep, nr_el)) + 1j * rng.standard_normal((nw, nw, nm, nr_ep, nr_el))
    ph = O.epmat_el_to_ph(el.reshape(-1, nr_el, order="F"), nw, nm, nr_el, nr_ep)
    want = el.transpose(0, 1, 2, 4, 3).reshape(-1, nr_ep, order="F")
    assert np.array_equal(ph, want)


def test_oracle_loop_orders_agree():
    """Both loop orders of the reference give the same ep (test/test_epmat.jl:45-80)."""
    m = _model()
    nw, nm = m.nw, m.nmodes
    ep = m.epmat
    nr_el, nr_ep = ep.irvec.shape[0], ep.irvec_next.shape[0]
    op_ph = O.epmat_el_to_ph(ep.op_r, nw, nm, nr_el, nr_ep)
    xk = np.array([0.1, -0.4, 0.7])
    xq = np.array([0.5, 0.2, -0.5])
    ham = m.el_ham
    hk = O.fourier_batched(ham.op_r, ham.ndata, ham.irvec, np.stack([xk, xk + xq], 1)).reshape(nw, nw, 2, order="F")
    _, U = O.eigen_batched(hk)
    w, uph = O.ph_eigen_batched(xq.reshape(3, 1), m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    uk, ukq = U[:, 1:4, 0], U[:, 0:3, 1]
    ref = _outer_k(m, xk, xq, uk, ukq, uph[:, :, 0])
    gRq = O.get_eph_RR_to_Rq(op_ph, ep.irvec_next, nw, nm, nr_el, xq, uph[:, :, 0])
    got = O.get_eph_Rq_to_kq_batched(gRq, ep.irvec, xk.reshape(3, 1), uk[:, :, None], ukq[:, :, None], nm)[..., 0]
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.abs(ref).max()


@pytest.fixture(scope="module")
def B(gpu_lib):
    from epb200 import batched

    return batched


def _dev_obj(irvec, op, irvec_next=None):
    from epb200.wannier import WannierObject, to_device

    return to_device(WannierObject(irvec, op, irvec_next=irvec_next))


@pytest.mark.gpu
@pytest.mark.parametrize("nw,nm", [(4, 6), (3, 2), (16, 12)])
def test_el_to_ph_bit_exact(B, nw, nm):
    m = synth.config2_model(seed=nw + nm, n_el=1, n_ph=1, nw=nw, natom=nm // 3 if nm % 3 == 0 else 1)
    ep = m.epmat
    nm = ep.op_r.shape[0] // (nw * nw * ep.irvec_next.shape[0])
    nr_el, nr_ep = ep.irvec.shape[0], ep.irvec_next.shape[0]
    ph = B.epmat_el_to_ph(_dev_obj(ep.irvec, ep.op_r, ep.irvec_next), nw, nm)
    assert np.array_equal(ph.irvec, ep.irvec_next) and np.array_equal(ph.irvec_next, ep.irvec)
    got = B.host(ph.op_r)
    assert np.array_equal(got, O.epmat_el_to_ph(ep.op_r, nw, nm, nr_el, nr_ep))


@pytest.mark.gpu
@pytest.mark.parametrize("nq", [1, 7, 40])
def test_RR_to_Rq(B, nq):
    m = _model(seed=20 + nq)
    nw, nm = m.nw, m.nmodes
    ep = m.epmat
    nr_el, nr_ep = ep.irvec.shape[0], ep.irvec_next.shape[0]
    xq = synth.random_kpoints(nq, nq)
    w, uph = O.ph_eigen_batched(xq, m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    ph = B.epmat_el_to_ph(_dev_obj(ep.irvec, ep.op_r, ep.irvec_next), nw, nm)
    import torch

    out = B.jl_empty((nw * nw * nm, nr_el, nq), torch.complex128)
    B.get_eph_RR_to_Rq_batched(out, B.get_interpolator(ph), xq, B.jl(uph))
    got = B.host(out)
    op_ph = O.epmat_el_to_ph(ep.op_r, nw, nm, nr_el, nr_ep)
    for iq in range(nq):
        ref = O.get_eph_RR_to_Rq(op_ph, ep.irvec_next, nw, nm, nr_el, xq[:, iq], uph[:, :, iq])
        np.testing.assert_allclose(got[:, :, iq], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("nw,nbk,nbkq,nk", [(4, 4, 4, 33), (4, 2, 3, 5), (8, 5, 8, 300), (16, 16, 16, 17)])
def test_Rq_to_kq_batched(B, nw, nbk, nbkq, nk):
    """Slice by slice against the per-k form (test/test_gpu.jl:92-107), g2 fold included."""
    rng = np.random.default_rng(nw * 100 + nk)
    nm = 6
    irvec_el = synth.irvec_box(2)
    g = np.asfortranarray(rng.random((nw * nw * nm, irvec_el.shape[0])) + 1j * rng.random((nw * nw * nm, irvec_el.shape[0])))
    xk = rng.random((3, nk)) * 2 - 0.5
    uks = np.asfortranarray(rng.random((nw, nbk, nk)) + 1j * rng.random((nw, nbk, nk)))
    ukqs = np.asfortranarray(rng.random((nw, nbkq, nk)) + 1j * rng.random((nw, nbkq, nk)))
    omega = rng.random(nm) + 0.1
    import torch

    ep = B.jl_empty((nbkq, nbk, nm, nk), torch.complex128)
    g2 = B.jl_empty((nbkq, nbk, nm, nk), torch.float64)
    gd = B.jl(g)
    B.get_eph_Rq_to_kq_batched(ep, gd, irvec_el, xk, B.jl(uks), B.jl(ukqs), g2_out=g2,
                               omega=torch.as_tensor(omega, device="cuda"))
    got, got2 = B.host(ep), B.host(g2)
    ref = O.get_eph_Rq_to_kq_batched(g, irvec_el, xk, uks, ukqs, nm)
    for k in range(nk):
        gk = O.get_fourier(g, g.shape[0], irvec_el, xk[:, k]).reshape(nw, nw, nm, order="F")
        per_k = np.einsum("im,ija,jn->mna", ukqs[:, :, k].conj(), gk, uks[:, :, k])
        np.testing.assert_allclose(got[..., k], per_k, rtol=1e-9, atol=1e-12 * np.abs(per_k).max())
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_allclose(got2, np.abs(ref) ** 2 / (2 * omega[None, None, :, None]), rtol=1e-11,
                               atol=1e-12 * (np.abs(ref) ** 2).max())


@pytest.mark.gpu
def test_outer_q_equals_outer_k_on_device(B):
    """The two loop orders on the device give the same ep (test/test_epmat.jl:45-80), for a k list."""
    import torch

    m = _model(seed=31, nw=8, natom=2)
    nw, nm = m.nw, m.nmodes
    ep = m.epmat
    nr_el = ep.irvec.shape[0]
    nk = 24
    xk = synth.random_kpoints(nk, 5)
    xq = synth.random_kpoints(1, 6)
    ham = m.el_ham
    hk = O.fourier_batched(ham.op_r, ham.ndata, ham.irvec, np.concatenate([xk, xk + xq], 1)).reshape(nw, nw, -1, order="F")
    _, U = O.eigen_batched(hk)
    uks, ukqs = np.asfortranarray(U[:, 2:6, :nk]), np.asfortranarray(U[:, 1:7, nk:])
    w, uph = O.ph_eigen_batched(xq, m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    # outer q on the device
    ph = B.epmat_el_to_ph(_dev_obj(ep.irvec, ep.op_r, ep.irvec_next), nw, nm)
    gRq = B.jl_empty((nw * nw * nm, nr_el, 1), torch.complex128)
    B.get_eph_RR_to_Rq_batched(gRq, B.get_interpolator(ph), xq, B.jl(uph))
    out = B.jl_empty((6, 4, nm, nk), torch.complex128)
    B.get_eph_Rq_to_kq_batched(out, gRq[0], ep.irvec, xk, B.jl(uks), B.jl(ukqs))
    got = B.host(out)
    for k in range(nk):
        ref = _outer_k(m, xk[:, k], xq[:, 0], uks[:, :, k], ukqs[:, :, k], uph[:, :, 0])
        np.testing.assert_allclose(got[..., k], ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
def test_outerq_edge_cases(B):
    import torch

    from epb200._lib import EpbError

    nw, nm = 4, 3
    irvec_el = synth.irvec_box(1)
    g = B.jl(np.ones((nw * nw * nm, irvec_el.shape[0]), dtype=np.complex128))
    ep = B.jl_empty((nw, nw, nm, 0), torch.complex128)
    empty = B.jl(np.zeros((nw, nw, 0), dtype=np.complex128))
    B.get_eph_Rq_to_kq_batched(ep, g, irvec_el, np.zeros((3, 0)), empty, empty)  # nk = 0 is a no-op
    from epb200 import _lib

    with pytest.raises(EpbError):  # nbk > nw
        _lib.check(_lib.lib().epb_eph_Rq_to_kq(_lib.default_context().h, _lib.ptr(g), nw, nm,
                                               _lib.RSet(_lib.default_context(), irvec_el).h, 0, 1, 0, nw + 1, 0, nw,
                                               0, 0, 0, 0))
    with pytest.raises(EpbError):  # g2 without omega
        out = B.jl_empty((nw, nw, nm, 1), torch.float64)
        _lib.check(_lib.lib().epb_eph_Rq_to_kq(_lib.default_context().h, _lib.ptr(g), nw, nm,
                                               _lib.RSet(_lib.default_context(), irvec_el).h, _lib.ptr(out), 1,
                                               _lib.ptr(out), nw, _lib.ptr(out), nw, 0, 0, _lib.ptr(out), 0))


# ---- the batched outer-q loop (run_eph_over_q_and_k) ---------------------------------------------
def _outer_k_record(m, xk, xq, window_k, window_kq):
    """The same gauge-invariant record through the outer-k chain (RR->kR, kR->kq)."""
    nw, nm = m.nw, m.nmodes
    ham = m.el_ham
    A = np.zeros(xq.shape[1])
    for iq in range(xq.shape[1]):
        x2 = np.concatenate([xk, xk + xq[:, iq:iq + 1]], 1)
        hk = O.fourier_batched(ham.op_r, ham.ndata, ham.irvec, x2).reshape(nw, nw, -1, order="F")
        E, U = O.eigen_batched(hk)
        _, uph = O.ph_eigen_batched(xq[:, iq:iq + 1], m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
        nk = xk.shape[1]
        for k in range(nk):
            s, t = O.inside_window(E[:, k], *window_k)
            s2, t2 = O.inside_window(E[:, nk + k], *window_kq)
            if t < s or t2 < s2:
                continue
            e = _outer_k(m, xk[:, k], xq[:, iq], U[:, s - 1:t, k], U[:, s2 - 1:t2, nk + k], uph[:, :, 0])
            A[iq] += np.sum(np.abs(e) ** 2)
    return A


def test_oracle_outer_q_record_matches_outer_k():
    m = _model(seed=41, nw=8)
    xk = synth.random_kpoints(12, 1)
    xq = synth.random_kpoints(3, 2)
    win_k, win_kq = (-5.0, 3.0), (-8.0, 6.0)
    A = O.outer_q_record(m, xk, xq, window_k=win_k, window_kq=win_kq)
    B = _outer_k_record(m, xk, xq, win_k, win_kq)
    assert np.all(A > 0)
    np.testing.assert_allclose(A, B, rtol=1e-11)


@pytest.fixture(scope="module")
def P(gpu_lib):
    from epb200 import outer_q, pipeline

    return outer_q, pipeline


class _Record:
    """The record calculator of test/test_gpu.jl:589-654 on the payload: per q, sum wtk |ep|^2."""

    def __init__(self, nq):
        import torch

        self.A = np.zeros(nq)
        self.acc = None
        self.begins = self.ends = 0
        self.widths = []
        self.torch = torch

    def begin_q(self, iq):
        self.begins += 1
        self.acc = self.torch.zeros((), dtype=self.torch.float64, device="cuda")

    def run_batch(self, p):
        self.widths.append(p.nk)
        self.acc += (p.eps.abs() ** 2 * p.wtk.view(-1, 1, 1, 1)).sum()

    def end_q(self, iq):
        self.ends += 1
        self.A[iq] = float(self.acc)


@pytest.mark.gpu
@pytest.mark.parametrize("basis,nw", [("eigenmode", 8), ("cartesian", 8), ("eigenmode", 20)])
def test_outer_q_loop_fp64(P, basis, nw):
    """Record A[iq] vs the oracle's per-point outer-q chain (rtol 1e-10; the reference's CPU-vs-GPU bar is
    1e-8, test/test_gpu.jl:673), with windows on both sides and weights. nw = 20 takes the per-mode
    rotation kernel (the staged one covers nw <= 16)."""
    outer_q, pipeline = P
    m = _model(seed=41, nw=nw)
    xk = synth.random_kpoints(37, 1)
    xq = synth.random_kpoints(4, 2)
    wtk = np.random.default_rng(0).random(37)
    win_k, win_kq = (0.0, 1.5), (-8.0, 6.0)
    dm = pipeline.DeviceModel(m)
    A, st = outer_q.run_eph_over_q_and_k(dm, xk, xq, wtk=wtk, window_k=win_k, window_kq=win_kq,
                                         eph_phonon_basis=basis)
    ref = O.outer_q_record(m, xk, xq, wtk=wtk, window_k=win_k, window_kq=win_kq, phonon_basis=basis)
    assert 0 < st["kept_k"] <= 37
    np.testing.assert_allclose(A, ref, rtol=1e-10)


@pytest.mark.gpu
def test_outer_q_loop_partial_batches_and_payload(P):
    """A partial final k batch (nk_batch_max below nk, test/test_gpu.jl:707-715) and a q chunk of 2 give
    the same record; the Python record calculator over the payload agrees; payload invariants hold."""
    import torch

    outer_q, pipeline = P
    m = _model(seed=43, nw=8)
    nk, nq = 29, 5
    xk = synth.random_kpoints(nk, 3)
    xq = synth.random_kpoints(nq, 4)
    win_k, win_kq = (0.0, 1.5), (-7.0, 5.0)
    dm = pipeline.DeviceModel(m)
    A0, st0 = outer_q.run_eph_over_q_and_k(dm, xk, xq, window_k=win_k, window_kq=win_kq)
    rec = _Record(nq)
    seen = {}

    class Check:
        def run_batch(self, p):
            assert p.eps.shape == (p.nk, m.nmodes, m.nw, m.nw)
            ik = p.ik.cpu().numpy()
            assert np.all((ik >= 0) & (ik < nk))
            np.testing.assert_allclose(p.xks.cpu().numpy().T, xk[:, ik], atol=0)
            ekq, ukq = p.ekq.cpu().numpy().T, p.ukq.cpu().numpy().T  # (nw, nk), (nw, nw, nk)
            out = (ekq < win_kq[0]) | (ekq > win_kq[1])
            for j in range(p.nk):
                assert np.all(ukq[:, out[:, j], j] == 0)
            seen.setdefault(p.iq, 0)
            seen[p.iq] += p.nk

    A1, st1 = outer_q.run_eph_over_q_and_k(dm, xk, xq, window_k=win_k, window_kq=win_kq, calculators=[rec, Check()],
                                           nk_batch_max=10, q_chunk=2)
    torch.cuda.synchronize()
    assert st1["k_batch"] == 10 and st1["q_chunk"] == 2
    assert rec.begins == nq and rec.ends == nq
    assert all(v == st1["kept_k"] for v in seen.values()) and len(seen) == nq
    assert st1["kept_k"] == 13 and sorted(set(rec.widths)) == [3, 10]
    np.testing.assert_allclose(A1, A0, rtol=1e-12)
    np.testing.assert_allclose(rec.A, A0, rtol=1e-12)
    ref = O.outer_q_record(m, xk, xq, window_k=win_k, window_kq=win_kq)
    np.testing.assert_allclose(A0, ref, rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("nw,nk,kb", [(16, 300, 0), (16, 700, 200), (20, 130, 0)])
def test_outer_q_loop_mixed(P, nw, nk, kb):
    """Mixed precision (split-BF16 H(k+q) and g(k, q), FP32 + FP64-refined eigensolves): record within 1e-5
    relative of FP64 (the |g|^2 bar of the mixed path); several k batches (rounded to 256 here) and the
    nw > 16 rotation included."""
    from epb200._lib import PREC_MIXED

    outer_q, pipeline = P
    m = synth.config2_model(seed=44, n_el=2, n_ph=1, nw=nw, natom=4)
    xk = synth.random_kpoints(nk, 5)
    xq = synth.random_kpoints(3, 6)
    dm = pipeline.DeviceModel(m)
    A64, _ = outer_q.run_eph_over_q_and_k(dm, xk, xq, window_k=(-5.0, 5.0), window_kq=(-8.0, 8.0))
    A32, st = outer_q.run_eph_over_q_and_k(dm, xk, xq, window_k=(-5.0, 5.0), window_kq=(-8.0, 8.0), prec=PREC_MIXED,
                                           nk_batch_max=kb)
    if kb:
        assert st["k_batch"] == 256 and st["batches"] == 3 * -(-st["kept_k"] // 256)
    assert np.max(np.abs(A32 - A64) / np.abs(A64)) <= 1e-5


@pytest.mark.gpu
def test_outer_q_loop_errors(P):
    """A calculator that raises aborts the loop with its exception; the context stays usable; an empty
    k window or an empty k list gives zeros; a calculator without run_batch is rejected up front."""
    outer_q, pipeline = P
    m = _model(seed=45, nw=4)
    xk = synth.random_kpoints(8, 7)
    xq = synth.random_kpoints(2, 8)
    dm = pipeline.DeviceModel(m)

    class Boom:
        def run_batch(self, p):
            raise RuntimeError("calculator failure")

    with pytest.raises(RuntimeError, match="calculator failure"):
        outer_q.run_eph_over_q_and_k(dm, xk, xq, calculators=[Boom()])
    with pytest.raises(TypeError):
        outer_q.run_eph_over_q_and_k(dm, xk, xq, calculators=[object()])
    A, st = outer_q.run_eph_over_q_and_k(dm, xk, xq, window_k=(100.0, 200.0))
    assert st["kept_k"] == 0 and np.all(A == 0)
    A, st = outer_q.run_eph_over_q_and_k(dm, np.zeros((3, 0)), xq)
    assert np.all(A == 0)
    A, st = outer_q.run_eph_over_q_and_k(dm, xk, xq)
    ref = O.outer_q_record(m, xk, xq)
    np.testing.assert_allclose(A, ref, rtol=1e-10)
