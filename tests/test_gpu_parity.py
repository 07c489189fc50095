"""GPU parity: every entry point, called through the C ABI, against the FP64 oracle.

Tolerances (stated per test) follow the reference's own: batched vs per-point rtol 1e-10 on CPU and
1e-9 on GPU (test/test_gpu.jl:120-122,342), phase <= 4 eps (test_gpu.jl:127-144), k+q identity
1e-13 (test_gpu.jl:156-211), eigenvalues vs LAPACK (test_gpu.jl:311-339).
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


def _rand_irvec(rng, n, lo=-2, hi=2):
    r = rng.integers(lo, hi + 1, size=(n, 3))
    return r[np.lexsort((r[:, 0], r[:, 1], r[:, 2]))]


def _cr(rng, *shape):
    return np.asfortranarray(rng.random(shape) + 1j * rng.random(shape))


def _dev_obj(irvec, op, irvec_next=None, ndata=None):
    from epb200.wannier import WannierObject, to_device

    return to_device(WannierObject(irvec, op, irvec_next=irvec_next, ndata=ndata))


def test_fourier_phase(B):
    rng = np.random.default_rng(1)
    irvec = rng.integers(-3, 4, size=(37, 3))
    xk = rng.random((3, 11))
    ph = B.host(B.fourier_phase(irvec, xk))
    assert np.max(np.abs(ph - O.fourier_phase(irvec, xk))) <= 4 * np.finfo(float).eps


@pytest.mark.parametrize("ndata,nr,nk,rmax", [(64, 343, 300, 3), (256, 729, 129, 4), (7, 20, 5, 2), (100, 50, 70, 20)])
def test_fourier_fp64(B, ndata, nr, nk, rmax):
    rng = np.random.default_rng(ndata + nr)
    if rmax <= 4 and nr == (2 * rmax + 1) ** 3:
        irvec = synth.irvec_box(rmax)
    else:
        irvec = _rand_irvec(rng, nr, -rmax, rmax)  # rmax=20 exercises the direct-phase path
    op = _cr(rng, ndata + 3, nr)
    obj = _dev_obj(irvec, op, ndata=ndata)
    xk = rng.random((3, nk)) * 2 - 0.5
    out = B.host(B.get_fourier_batched(B.get_interpolator(obj), xk))
    ref = O.fourier_batched(op, ndata, irvec, xk)
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def _herm_stack(rng, n, nk):
    a = rng.standard_normal((n, n, nk)) + 1j * rng.standard_normal((n, n, nk))
    return np.asfortranarray((a + a.conj().transpose(1, 0, 2)) / 2)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n", [1, 3, 4, 8, 16, 17, 32, 40, 64])
def test_eigh_batched(B, n, prec):
    rng = np.random.default_rng(n)
    nk = 67
    h = _herm_stack(rng, n, nk)
    E, U = B.eigen_batched(B.jl(h), prec=prec)
    E, U = B.host(E), B.host(U)
    eref = O.eigvals_batched(h.copy())
    scale = np.abs(eref).max()
    # FP64: LAPACK-level agreement; mixed: FP32 solve + FP64 refinement reaches the same level
    tol = 1e-12 if prec == 0 else 1e-11
    assert np.max(np.abs(E - eref)) <= tol * scale
    for k in range(nk):
        rec = U[:, :, k] @ np.diag(E[:, k]) @ U[:, :, k].conj().T
        assert np.max(np.abs(rec - h[:, :, k])) <= 10 * tol * scale
        assert np.max(np.abs(U[:, :, k].conj().T @ U[:, :, k] - np.eye(n))) <= 10 * tol * n
    ev = B.host(B.eigvals_batched(B.jl(h), prec=prec))
    assert np.max(np.abs(ev - eref)) <= tol * scale


@pytest.mark.parametrize("n", [8, 16, 32, 96])
def test_eigh_clusters_stress(B, n):
    """Every instance with planted 2-4-fold clusters spaced 1e-10 (thousands for the register-resident
    n <= 16 solver, where a first-order refinement range that was too wide once left 0.5 % of such
    matrices with non-orthogonal cluster vectors): eigenvalues to 1e-11 and U diag(E) U^H to 1e-10 of the
    largest |eigenvalue|, FP32 solve + FP64 refinement."""
    count = 2400 if n <= 16 else 300
    ns, mats = synth.config3_matrices(count, seed=101 + n, sizes=[n], degenerate_frac=1.0)
    h = np.asfortranarray(np.stack(mats, axis=-1))
    E, U = B.eigen_batched(B.jl(h), prec=1)
    E, U = B.host(E), B.host(U)
    eref = O.eigvals_batched(h.copy())
    scale = np.abs(eref).max()
    assert np.max(np.abs(E - eref)) <= 1e-11 * scale
    rec = np.einsum("ijk,jk,ljk->ilk", U, E, U.conj())
    assert np.max(np.abs(rec - h)) <= 1e-10 * scale


def test_eigh_degenerate_clusters(B):
    """Planted 2-4-fold clusters spaced 1e-10: eigenvalues and the cluster projectors match."""
    ns, mats = synth.config3_matrices(200, seed=7, sizes=[8, 16, 24], degenerate_frac=1.0)
    for prec in (0, 1):
        for n in (8, 16, 24):
            sel = [m for k, m in zip(ns, mats) if k == n]
            h = np.asfortranarray(np.stack(sel, axis=-1))
            E, U = B.eigen_batched(B.jl(h), prec=prec)
            E, U = B.host(E), B.host(U)
            eref = O.eigvals_batched(h.copy())
            assert np.max(np.abs(E - eref)) <= 1e-11 * np.abs(eref).max()
            for k in range(h.shape[2]):
                rec = U[:, :, k] @ np.diag(E[:, k]) @ U[:, :, k].conj().T
                assert np.max(np.abs(rec - h[:, :, k])) <= 1e-10 * np.abs(eref).max()


def test_phonon_eigen(B):
    m = synth.config2_model(seed=3, n_el=1, n_ph=2, nw=4, natom=4, with_epmat=False)
    xq = synth.random_kpoints(50, 9)
    itp = B.get_interpolator(_dev_obj(m.ph_dyn.irvec, m.ph_dyn.op_r))
    w_ref, u_ref = O.ph_eigen_batched(xq, m.ph_dyn.op_r, m.ph_dyn.irvec, m.mass)
    for prec in (0, 1):
        w, u = B.ph_eigen_batched(itp, xq, m.mass, prec=prec)
        w, u = B.host(w), B.host(u)
        np.testing.assert_allclose(w, w_ref, rtol=1e-10)
        # gauge-invariant: sum_nu u[:, nu] w_nu^2 u[:, nu]^dagger (mass weighted) reproduces D/m
        sm = np.sqrt(m.mass)
        for q in range(0, 50, 7):
            us = u[:, :, q] * sm[:, None]
            ur = u_ref[:, :, q] * sm[:, None]
            a = us @ np.diag(w[:, q] ** 2) @ us.conj().T
            b = ur @ np.diag(w_ref[:, q] ** 2) @ ur.conj().T
            np.testing.assert_allclose(a, b, atol=1e-10 * np.abs(b).max())


def _eph_setup(rng, nwe=3, nm=4, nr_el=20, nr_ep=15, nk=5, nq=6, nband=None):
    nband = nwe if nband is None else nband
    irvec_el, irvec_ep = _rand_irvec(rng, nr_el), _rand_irvec(rng, nr_ep)
    op = _cr(rng, nwe * nwe * nm * nr_ep, nr_el)
    return dict(irvec_el=irvec_el, irvec_ep=irvec_ep, op=op, ks=rng.random((3, nk)), qs=rng.random((3, nq)),
                uks=_cr(rng, nwe, nband, nk), uphs=_cr(rng, nm, nm, nq), ukqs=_cr(rng, nwe, nband, nq),
                nwe=nwe, nm=nm, nr_ep=nr_ep, nband=nband)


@pytest.mark.parametrize("nwe,nm,nband", [(3, 4, 3), (6, 6, 4), (16, 12, 16)])
def test_eph_batched_drivers(B, nwe, nm, nband):
    """test/test_gpu.jl:44-122 on the device: RR->kR, kR->kq, g2 vs per-point oracle, rtol 1e-9."""
    import torch

    rng = np.random.default_rng(nwe * 10 + nm)
    f = _eph_setup(rng, nwe=nwe, nm=nm, nband=nband, nr_el=27 if nwe < 16 else 30)
    obj = _dev_obj(f["irvec_el"], f["op"], irvec_next=f["irvec_ep"])
    itp = B.get_interpolator(obj)
    nk, nq = f["ks"].shape[1], f["qs"].shape[1]
    out = B.jl_empty((nwe * nband * nm, f["nr_ep"], nk), torch.complex128)
    B.get_eph_RR_to_kR_batched(out, itp, f["ks"], B.jl(f["uks"]))
    out_h = B.host(out)
    refs = [O.get_eph_RR_to_kR(f["op"], f["irvec_el"], f["nr_ep"], nwe, nm, f["ks"][:, k], f["uks"][:, :, k])
            for k in range(nk)]
    for k in range(nk):
        np.testing.assert_allclose(out_h[:, :, k], refs[k], rtol=1e-9, atol=1e-12 * np.abs(refs[k]).max())
    # kR -> kq with the phase-taking method, plus the g2 fold
    phase = B.fourier_phase(f["irvec_ep"], f["qs"])
    omega = rng.random((nm, nq)) + 0.5
    ep = B.jl_empty((nband, nband, nm, nq), torch.complex128)
    g2 = B.jl_empty((nband, nband, nm, nq), torch.float64)
    kR0 = B.jl(refs[0])
    B.get_eph_kR_to_kq_batched(ep, kR0, phase, B.jl(f["uphs"]), B.jl(f["ukqs"]), g2_out=g2, omega=B.jl(omega))
    ep_ref = np.stack([O.get_eph_kR_to_kq(refs[0], f["irvec_ep"], f["qs"][:, q], f["uphs"][:, :, q],
                                          f["ukqs"][:, :, q], nband) for q in range(nq)], axis=-1)
    np.testing.assert_allclose(B.host(ep), ep_ref, rtol=1e-9, atol=1e-12 * np.abs(ep_ref).max())
    g2_ref = np.abs(ep_ref) ** 2 / (2 * omega[None, None])
    np.testing.assert_allclose(B.host(g2), g2_ref, rtol=1e-9, atol=1e-12 * g2_ref.max())


def test_kq_convention_identity_gpu(B):
    """test/test_gpu.jl:156-211 on the device: k+q convention == q convention, rtol 1e-13."""
    import torch

    rng = np.random.default_rng(5)
    nwe, nm, nr_el, nr_ep, nq = 3, 4, 12, 15, 9
    f = _eph_setup(rng, nwe=nwe, nm=nm, nr_el=nr_el, nr_ep=nr_ep, nk=1, nq=nq)
    xk = np.array([[0.75], [-0.40], [0.35]])
    xkqs = rng.integers(-10, 11, size=(3, nq)) / 20.0
    qs = np.mod(xkqs - xk, 1.0)
    itp = B.get_interpolator(_dev_obj(f["irvec_el"], f["op"], irvec_next=f["irvec_ep"]))
    ndata = nwe * nwe * nm
    kR = B.jl_empty((ndata, nr_ep, 1), torch.complex128)
    B.get_eph_RR_to_kR_batched(kR, itp, xk, B.jl(f["uks"][:, :, :1]))
    ref = B.jl_empty((nwe, nwe, nm, nq), torch.complex128)
    B.get_eph_kR_to_kq_batched(ref, kR[0], B.fourier_phase(f["irvec_ep"], qs), B.jl(f["uphs"]), B.jl(f["ukqs"]))
    pmk = torch.conj_physical(B.fourier_phase(f["irvec_ep"], xk))
    kR2 = B.jl_empty((ndata, nr_ep, 1), torch.complex128)
    B.get_eph_RR_to_kR_batched(kR2, itp, xk, B.jl(f["uks"][:, :, :1]), additional_phase=pmk)
    out = B.jl_empty((nwe, nwe, nm, nq), torch.complex128)
    B.get_eph_kR_to_kq_batched(out, kR2[0], B.fourier_phase(f["irvec_ep"], xkqs), B.jl(f["uphs"]), B.jl(f["ukqs"]))
    np.testing.assert_allclose(B.host(out), B.host(ref), rtol=1e-13, atol=1e-13 * np.abs(B.host(ref)).max())


def test_window_filter_exact(B):
    rng = np.random.default_rng(9)
    nw, nk = 16, 5000
    E = np.sort(rng.standard_normal((nw, nk)) * 3, axis=0)
    E[:, 7] = 0.25  # degenerate values at the window edge
    E[3, 11] = 0.25
    E = np.sort(E, axis=0)  # the contract is sorted energies per k
    wmin, wmax = -0.1, 0.25
    bmin, bmax, keep, nbelow = B.window_filter(B.jl(np.asfortranarray(E)), wmin, wmax)
    ref = O.filter_kpoints(E, np.ones(nk), wmin, wmax)
    assert np.array_equal(bmin.cpu().numpy(), ref["band_min_per_k"])
    assert np.array_equal(bmax.cpu().numpy(), ref["band_max_per_k"])
    assert np.array_equal(keep.cpu().numpy(), np.nonzero(ref["ik_keep"])[0])
    assert float(nbelow.sum()) == ref["nelec_below_window"]
    # empty input and an all-out window
    _, _, keep0, _ = B.window_filter(B.jl(np.asfortranarray(E)), 100.0, 101.0)
    assert keep0.numel() == 0


def test_filtered_states_device_indmap(B):
    """Device FilteredStates from the window filter's band ranges, bit-exact against the oracle's
    filtered_states_indmap (band_states.jl:99-121) embedded in physical band rows as the device calculators
    read it (_indmap_to_device, band_states.jl:283-287): several blocks of k, an all-out window, and a
    state-list capacity below the state count (the map stays complete)."""
    rng = np.random.default_rng(19)
    nw, nk = 16, 5000
    E = np.sort(rng.standard_normal((nw, nk)) * 3, axis=0)
    wmin, wmax = -0.5, 0.9
    bmin, bmax, keep, _ = B.window_filter(B.jl(np.asfortranarray(E)), wmin, wmax)
    indmap, iks, ibands, n, ign, nband = B.filtered_states(bmin, bmax, nw)
    ref = O.filter_kpoints(E, np.ones(nk), wmin, wmax)
    riks, ribs, rmap, rign = O.filtered_states_indmap(ref["ik_keep"], ref["band_min_per_k"], ref["band_max_per_k"])
    assert n == len(riks) > 0 and ign == rign and nband == rmap.shape[0]
    assert np.array_equal(iks.cpu().numpy(), riks) and np.array_equal(ibands.cpu().numpy(), ribs)
    phys = np.zeros((nw, nk), dtype=np.int64)
    phys[rign:rign + rmap.shape[0], :] = rmap
    assert np.array_equal(B.host(indmap), phys)
    # capacity below n: identical map, the first `cap` states only
    indmap2, iks2, ibands2, n2, _, _ = B.filtered_states(bmin, bmax, nw, capacity=n // 3)
    assert n2 == n and np.array_equal(B.host(indmap2), phys)
    assert np.array_equal(iks2.cpu().numpy(), riks[: n // 3]) and np.array_equal(ibands2.cpu().numpy(), ribs[: n // 3])
    # nothing in the window
    b0, b1, _, _ = B.window_filter(B.jl(np.asfortranarray(E)), 100.0, 101.0)
    indmap0, iks0, _, n0, ign0, nband0 = B.filtered_states(b0, b1, nw)
    assert (n0, ign0, nband0) == (0, 0, 0) and iks0.numel() == 0 and not B.host(indmap0).any()


def test_fill_iqs_vs_oracle(B):
    import torch

    for ngrid, shift in [((4, 4, 4), (0, 0, 0)), ((4, 3, 5), (0.5 / 4, 0, 0.5 / 5))]:
        k = synth.grid_kpoints(ngrid)
        kq = synth.grid_kpoints(ngrid, shift)
        dense = np.zeros(int(np.prod(ngrid)), dtype=np.int64)
        for iq in range(kq.shape[1]):
            dense[O.hash_xk(kq[:, iq], ngrid, shift)] = iq + 1
        kq_int = np.stack([O.grid_coords_reduced(kq[:, j], ngrid, shift) for j in range(kq.shape[1])], 1)
        dev_kq = torch.from_numpy(np.ascontiguousarray(kq_int.T)).cuda()
        dev_dense = torch.from_numpy(dense).cuda()
        for ik in range(0, k.shape[1], 7):
            k_int = O.grid_coords_reduced(k[:, ik], ngrid, (0, 0, 0))
            got = B.fill_iqs(dev_kq, k_int, ngrid, dev_dense).cpu().numpy()
            assert np.array_equal(got, O.fill_iqs(dense, ngrid, kq_int, k_int))
    # a miss raises (kq - k not in the q list)
    from epb200._lib import EpbError

    with pytest.raises(EpbError):
        B.fill_iqs(dev_kq, np.array([0, 0, 0]), ngrid, torch.zeros_like(dev_dense))


def test_error_paths(B):
    """Bad shapes and injected allocation failure return status codes, never crash."""
    from epb200 import _lib
    from epb200._lib import EpbError

    ctx = _lib.default_context()
    L = _lib.lib()
    assert L.epb_eigh_batched(ctx.h, None, 0, 1, None, b"V", 0) == _lib.EPB_ERR_ARG
    assert L.epb_eigh_batched(ctx.h, None, 4, 1, None, b"X", 0) == _lib.EPB_ERR_ARG
    rng = np.random.default_rng(0)
    big = _herm_stack(rng, 128, 2)
    with pytest.raises(EpbError):
        B.eigen_batched(B.jl(big))
    # injected OOM on the next workspace growth
    import torch

    c2 = _lib.Context(0)
    L.epb_debug_fail_alloc(c2.h, 1)
    irvec = synth.irvec_box(1)
    rs = _lib.RSet(c2, irvec)
    xk = B.jl(np.zeros((3, 4)))
    nrep = 20000
    op = torch.zeros((irvec.shape[0], 1), dtype=torch.complex128, device="cuda")
    out = torch.zeros((1, 1), dtype=torch.complex128, device="cuda")
    st = L.epb_eph_RR_to_kR(c2.h, op.data_ptr(), 1, 1, 1, rs.h, xk.data_ptr(), 4,
                            torch.zeros(16, dtype=torch.complex128, device="cuda").data_ptr(), 1, None,
                            torch.zeros(64, dtype=torch.complex128, device="cuda").data_ptr(), 0)
    assert st == _lib.EPB_ERR_OOM, L.epb_last_error()
    assert b"injected" in L.epb_last_error()
    del nrep, out
