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
