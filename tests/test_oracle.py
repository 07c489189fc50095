"""Oracle self-tests: each restates a known-answer or identity test of the reference.

These pin the CPU restatement (oracle/epb_oracle.py) to the reference's own test suite, because the
reference (Julia) cannot be run in this environment.
"""
import json
import os

import numpy as np
import pytest

from oracle import epb_oracle as O
from epb200 import synth
from epb200.wannier import WannierObject

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rand_irvec(rng, n, lo=-2, hi=2):
    r = rng.integers(lo, hi + 1, size=(n, 3))
    return r[np.lexsort((r[:, 0], r[:, 1], r[:, 2]))]


def test_fourier_phase_vs_scalar_cispi():
    """test/test_gpu.jl:127-144 -- phase vs scalar cispi(2 R.x), max error <= 4 eps."""
    rng = np.random.default_rng(11)
    nr, nk = 37, 11
    irvec = rng.integers(-3, 4, size=(nr, 3))
    xk = rng.random((3, nk))
    ph = O.fourier_phase(irvec, xk)
    import mpmath

    mpmath.mp.prec = 120
    ref = np.empty((nr, nk), dtype=complex)
    for i in range(nr):
        for j in range(nk):
            # the reference evaluates R.x in Float64 (same rounding), then an exact cispi
            t = (float(irvec[i, 0]) * xk[0, j] + float(irvec[i, 1]) * xk[1, j]) + float(irvec[i, 2]) * xk[2, j]
            a = mpmath.mpf(2.0 * t)
            ref[i, j] = complex(mpmath.cospi(a), mpmath.sinpi(a))
    assert np.max(np.abs(ph - ref)) <= 4 * np.finfo(float).eps


def _eph_fixture(rng, nwe=3, nmodes=4, nr_el=20, nr_ep=15, nk=5, nq=6):
    irvec_el = _rand_irvec(rng, nr_el)
    irvec_ep = _rand_irvec(rng, nr_ep)
    op = rng.random((nwe * nwe * nmodes * nr_ep, nr_el)) + 1j * rng.random((nwe * nwe * nmodes * nr_ep, nr_el))
    ks = rng.random((3, nk))
    qs = rng.random((3, nq))
    cr = lambda *s: rng.random(s) + 1j * rng.random(s)
    return dict(irvec_el=irvec_el, irvec_ep=irvec_ep, op=np.asfortranarray(op), ks=ks, qs=qs,
                uks=cr(nwe, nwe, nk), uphs=cr(nmodes, nmodes, nq), ukqs=cr(nwe, nwe, nq),
                nwe=nwe, nmodes=nmodes, nr_ep=nr_ep)


def test_batched_eph_drivers_vs_per_point():
    """test/test_gpu.jl:44-122 -- list-batched RR->kR, kR->kq and g2 vs per-k/q, rtol 1e-10."""
    rng = np.random.default_rng(12)
    f = _eph_fixture(rng)
    nwe, nm, nr_ep = f["nwe"], f["nmodes"], f["nr_ep"]
    nk, nq = f["ks"].shape[1], f["qs"].shape[1]
    refs = [O.get_eph_RR_to_kR(f["op"], f["irvec_el"], nr_ep, nwe, nm, f["ks"][:, k], f["uks"][:, :, k])
            for k in range(nk)]
    batched = O.get_eph_RR_to_kR_batched(f["op"], f["irvec_el"], nr_ep, nwe, nm, f["ks"], f["uks"])
    for k in range(nk):
        np.testing.assert_allclose(batched[:, :, k], refs[k], rtol=1e-10)
    ep_ref = np.stack([O.get_eph_kR_to_kq(refs[0], f["irvec_ep"], f["qs"][:, q], f["uphs"][:, :, q],
                                          f["ukqs"][:, :, q], nwe) for q in range(nq)], axis=-1)
    phase = O.fourier_phase(f["irvec_ep"], f["qs"])
    omega = rng.random((nm, nq)) + 0.5
    ep, g2 = O.get_eph_kR_to_kq_batched(refs[0], phase, f["uphs"], f["ukqs"], nwe, omega)
    np.testing.assert_allclose(ep, ep_ref, rtol=1e-10)
    np.testing.assert_allclose(g2, np.abs(ep_ref) ** 2 / (2 * omega[None, None]), rtol=1e-10)


def test_kq_convention_identity():
    """test/test_gpu.jl:156-211 -- the k+q convention (conj(e^{2 pi i Rp.xk}) folded into the kR
    object, transform at x_{k+q}) reproduces the q convention; q needs a mod-G reduction; rtol 1e-13."""
    rng = np.random.default_rng(14)
    nwe, nm, nr_el, nr_ep, nq = 3, 4, 12, 15, 9
    irvec_el, irvec_ep = _rand_irvec(rng, nr_el), _rand_irvec(rng, nr_ep)
    op = np.asfortranarray(rng.random((nwe * nwe * nm * nr_ep, nr_el)) + 1j * rng.random((nwe * nwe * nm * nr_ep, nr_el)))
    xk = np.array([0.75, -0.40, 0.35])
    xkqs = rng.integers(-10, 11, size=(3, nq)) / 20.0
    qs = np.mod(xkqs - xk[:, None], 1.0)
    assert np.any(qs != xkqs - xk[:, None])
    uk = rng.random((nwe, nwe, 1)) + 1j * rng.random((nwe, nwe, 1))
    uphs = rng.random((nm, nm, nq)) + 1j * rng.random((nm, nm, nq))
    ukqs = rng.random((nwe, nwe, nq)) + 1j * rng.random((nwe, nwe, nq))
    kR = O.get_eph_RR_to_kR_batched(op, irvec_el, nr_ep, nwe, nm, xk.reshape(3, 1), uk)[:, :, 0]
    ref, _ = O.get_eph_kR_to_kq_batched(kR, O.fourier_phase(irvec_ep, qs), uphs, ukqs, nwe)
    pmk = np.conj(O.fourier_phase(irvec_ep, xk.reshape(3, 1)))
    kR2 = O.get_eph_RR_to_kR_batched(op, irvec_el, nr_ep, nwe, nm, xk.reshape(3, 1), uk,
                                     additional_phase=pmk)[:, :, 0]
    out, _ = O.get_eph_kR_to_kq_batched(kR2, O.fourier_phase(irvec_ep, xkqs), uphs, ukqs, nwe)
    np.testing.assert_allclose(out, ref, rtol=1e-13)


def test_eigen_batched_reconstruction():
    """test/test_gpu.jl:260-273 -- eigenvalues vs LAPACK, U diag(E) U^dagger == H."""
    rng = np.random.default_rng(15)
    nw, nk = 8, 5
    a = rng.random((nw, nw, nk)) + 1j * rng.random((nw, nw, nk))
    h = (a + a.conj().transpose(1, 0, 2)) / 2
    e, u = O.eigen_batched(h.copy())
    for k in (0, 2, 4):
        np.testing.assert_allclose(np.sort(e[:, k]), np.linalg.eigvalsh(h[:, :, k]), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(u[:, :, k] @ np.diag(e[:, k]) @ u[:, :, k].conj().T, h[:, :, k], atol=1e-12)
    np.testing.assert_allclose(O.eigvals_batched(h.copy()), e, atol=1e-12)


def test_diagonalize_identities():
    """test/test_diagonalize.jl:18-48 -- electron values/vectors, phonon sign*sqrt and mass."""
    rng = np.random.default_rng(123)
    a = (rng.standard_normal((5, 5)) + 1j * rng.standard_normal((5, 5))) / np.sqrt(2)
    a = a + a.conj().T
    vals = np.linalg.eigvalsh(a)
    e, u = O.solve_eigen_el(a)
    np.testing.assert_allclose(e, vals, atol=1e-12)
    np.testing.assert_allclose(u * e[None, :], a @ u, atol=1e-12)
    mass = np.abs(rng.random(5)) + 1
    w, v = O.solve_eigen_ph(a, mass)
    np.testing.assert_allclose(w ** 2 * np.sign(w), vals, atol=1e-12)
    vs = v * np.sqrt(mass)[:, None]
    np.testing.assert_allclose(vs * (w ** 2 * np.sign(w))[None, :], a @ vs, atol=1e-12)


def test_epw_gauge_fix_degenerate():
    """src/diagonalize.jl:35-86 -- degenerate groups are rotated to diagonalise the EPW matrix."""
    rng = np.random.default_rng(16)
    n = 6
    q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ev = np.array([-1.0, 0.5, 0.5, 0.5 + 1e-9, 2.0, 3.0])
    h = (q * ev) @ q.conj().T
    h = (h + h.conj().T) / 2
    e, u = O.solve_eigen_el(h)
    p = O.degeneracy_perturbation_matrix(n)
    sub = u[:, 1:4].conj().T @ p @ u[:, 1:4]
    off = sub - np.diag(np.diag(sub))
    assert np.max(np.abs(off)) < 1e-10
    # rotation inside a group mixes levels split by < cutoff, so u^dagger H u is diagonal to ~1e-9
    np.testing.assert_allclose(u.conj().T @ h @ u, np.diag(e), atol=1e-8)


def test_inside_window_inclusive():
    """src/filter.jl:19 -- searchsortedfirst/last, inclusive on both ends."""
    e = np.array([-1.0, 0.0, 0.5, 0.5, 1.0, 2.0])
    assert O.inside_window(e, 0.0, 1.0) == (2, 5)
    assert O.inside_window(e, 0.1, 0.4) == (3, 2)           # empty
    assert O.inside_window(e, -np.inf, np.inf) == (1, 6)
    assert O.inside_window(e, 3.0, 4.0) == (7, 6)


def test_iq_hash_vs_xk_to_ik():
    """test/test_iq_build.jl:230-310 -- integer hash equals the float xk_to_ik, shifted grids."""
    for ngrid, shift in [((4, 4, 4), (0, 0, 0)), ((3, 5, 2), (0, 0, 0)), ((4, 3, 5), (0.5 / 4, 0, 0.5 / 5))]:
        k = synth.grid_kpoints(ngrid)
        kq = synth.grid_kpoints(ngrid, shift)
        q = synth.grid_kpoints(ngrid, shift)  # q = kq - k lives on the shifted grid
        dense = np.zeros(int(np.prod(ngrid)), dtype=np.int64)
        for iq in range(q.shape[1]):
            dense[O.hash_xk(q[:, iq], ngrid, shift)] = iq + 1
        kq_int = np.stack([O.grid_coords_reduced(kq[:, j], ngrid, shift) for j in range(kq.shape[1])], 1)
        for ik in range(k.shape[1]):
            k_int = O.grid_coords_reduced(k[:, ik], ngrid, (0, 0, 0))
            iqs = O.fill_iqs(dense, ngrid, kq_int, k_int)
            for j in range(kq.shape[1]):
                assert iqs[j] == dense[O.hash_xk(kq[:, j] - k[:, ik], ngrid, shift)]


def test_bte_increments_golden():
    """test/boltzmann/test_gpu_boltzmann_calculator.jl:5-29 -- pinned values, rtol 1e-12."""
    with open(os.path.join(GOLDEN, "bte_increments.json")) as fh:
        gold = json.load(fh)
    args = gold["input"]
    for m, (so_ref, si_ref) in gold["methods"].items():
        so, si = O.bte_scattering_increments(int(m), args["ek"], args["ekq"], args["wq"], args["g2"],
                                             args["wtq"], args["mu"], args["T"], args["eta"])
        assert so == pytest.approx(so_ref, rel=1e-12)
        assert si == pytest.approx(si_ref, rel=1e-12)
    assert O.bte_scattering_increments(5, 10.0, -10.0, 0.01, 1e-3, 1.0, 0.01, 0.01, 0.005) == (0.0, 0.0)


def test_synthetic_model_properties():
    """Generator invariants: H(-R) = H(R)^dagger, ASR, real positive phonon frequencies."""
    m = synth.config2_model(seed=5, n_el=2, n_ph=1, nw=4, natom=2)
    h = m.el_ham.op_r.reshape(4, 4, -1, order="F")
    idx = {tuple(r): i for i, r in enumerate(m.el_ham.irvec)}
    for i, r in enumerate(m.el_ham.irvec):
        np.testing.assert_allclose(h[:, :, idx[tuple(-r)]], h[:, :, i].conj().T)
    d = m.ph_dyn.op_r.reshape(6, 6, -1, order="F").real
    asr = d.sum(axis=2).reshape(2, 3, 2, 3).sum(axis=2)      # sum over R and b
    assert np.max(np.abs(asr)) < 1e-12
    w, _ = O.ph_eigen_batched(np.array([[0.0, 0.3], [0.0, 0.1], [0.0, 0.7]]), m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    assert np.all(w[3:, 0] > 0) and np.max(np.abs(w[:3, 0])) < 1e-6 and np.all(w[:, 1] > 0)


def test_eph_pairs_end_to_end_small():
    """q-convention pass (run_eph_over_k_and_q.jl semantics) agrees with the batched drivers."""
    m = synth.config2_model(seed=6, n_el=1, n_ph=1, nw=4, natom=1)
    xks = synth.random_kpoints(3, 1)
    xqs = synth.random_kpoints(4, 2)
    pairs = [(ik, iq) for ik in range(3) for iq in range(4)]
    res = O.eph_pairs(m, xks, xqs, pairs)
    # batched recomputation for ik = 1
    ham, ep = m.el_ham, m.epmat
    nw, nm = m.nw, m.nmodes
    hk = O.fourier_batched(ham.op_r, ham.ndata, ham.irvec, xks).reshape(nw, nw, -1, order="F")
    ek, uk = O.eigen_batched(hk)
    kR = O.get_eph_RR_to_kR_batched(ep.op_r, ep.irvec, ep.irvec_next.shape[0], nw, nm, xks, uk)
    xkq = xks[:, 1:2] + xqs
    hkq = O.fourier_batched(ham.op_r, ham.ndata, ham.irvec, xkq).reshape(nw, nw, -1, order="F")
    ekq, ukq = O.eigen_batched(hkq)
    w, uph = O.ph_eigen_batched(xqs, m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    _, g2 = O.get_eph_kR_to_kq_batched(kR[:, :, 1], O.fourier_phase(ep.irvec_next, xqs), uph, ukq, nw, w)
    for iq in range(4):
        r = res[1 * 4 + iq]
        np.testing.assert_allclose(r["g2"], g2[:, :, :, iq], rtol=1e-9)
