"""Host-side mirror of the reference's batched Wannier->Bloch API, backed by libepb200.so.

Names, argument meaning and error behaviour follow ElectronPhonon.jl:
  * get_interpolator / BatchedWannierInterpolator / get_fourier_batched
      (src/wannier/WannierInterpolator.jl:84-96, src/wannier/batched_interpolator.jl:39-73,200-214)
  * fourier_phase (src/wannier/batched_fourier_core.jl:24-30)
  * eigvals_batched / eigen_batched, get_el_eigen[_valueonly]_batched
      (src/wannier_to_bloch_batched.jl:30-105, ext/ElectronPhononCUDAExt.jl:80-115)
  * get_eph_RR_to_kR_batched / get_eph_kR_to_kq_batched / eph_apply_rotations
      (src/wannier_to_bloch_batched.jl:178-273,442-455)
  * epmat_el_to_ph / get_eph_RR_to_Rq_batched / get_eph_Rq_to_kq_batched, the outer-q loop
      (src/model_new.jl:551-565, src/wannier_to_bloch.jl:277-300, src/wannier_to_bloch_batched.jl:317-377)
  * window filter (src/filter.jl:19,40-100), fill_iqs (src/calculator/run_eph_over_k_and_kq.jl:565-582)

Device arrays are torch tensors holding the bytes of the Julia column-major array: a Julia array of
size (n1, n2, ..., nd) is a contiguous torch tensor of shape (nd, ..., n2, n1). `jl()` and
`host()` convert between Fortran-ordered numpy arrays and that layout. Assertion failures of the
reference become AssertionError here; library failures raise `EpbError`.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import PREC_FP64, PREC_MIXED, check, ptr  # noqa: F401
from .wannier import WannierObject


def _torch():
    import torch

    return torch


def jl(arr, device="cuda", dtype=None):
    """Fortran-ordered numpy array (Julia shape) -> device tensor in Julia byte layout."""
    torch = _torch()
    a = np.asfortranarray(arr if dtype is None else np.asarray(arr, dtype=dtype))
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device)


def host(t):
    """Device tensor in Julia byte layout -> Fortran-ordered numpy array with the Julia shape."""
    return t.detach().cpu().numpy().T


def jl_empty(shape, dtype, device="cuda"):
    torch = _torch()
    return torch.empty(tuple(reversed(shape)), dtype=dtype, device=device)


def _jlshape(t):
    return tuple(reversed(t.shape))


def _ctx():
    return _lib.default_context()


def _xk_dev(xks):
    """(3, nk) crystal coordinates -> device float64 tensor of the same bytes."""
    torch = _torch()
    if isinstance(xks, torch.Tensor):
        assert xks.dtype == torch.float64 and xks.is_cuda and xks.is_contiguous()
        return xks
    x = np.asfortranarray(np.asarray(xks, dtype=np.float64).reshape(3, -1))
    return jl(x)


# ---------------------------------------------------------------------------------------------
class BatchedWannierInterpolator:
    """Whole-batch Fourier engine over a device WannierObject (batched_interpolator.jl:39-73)."""

    def __init__(self, parent: WannierObject, batch_size: int | None = None):
        assert parent.on_device, "BatchedWannierInterpolator needs a device WannierObject (to_device)"
        self.parent = parent
        self.batch_size = batch_size
        self.rset = _lib.RSet(_ctx(), parent.irvec)


def get_interpolator(obj: WannierObject, fourier_mode: str = "batched", batch_size=None):
    if fourier_mode not in ("batched",):
        raise ValueError(f"fourier_mode={fourier_mode!r}: the device path implements 'batched'")
    return BatchedWannierInterpolator(obj, batch_size)


def fourier_phase(itp_or_irvec, xks):
    """phase (nr, nk) c128 on the device (batched_fourier_core.jl:24-30)."""
    torch = _torch()
    rset = itp_or_irvec.rset if isinstance(itp_or_irvec, BatchedWannierInterpolator) else _lib.RSet(_ctx(), itp_or_irvec)
    x = _xk_dev(xks)
    nk = x.numel() // 3
    out = jl_empty((rset.nr, nk), torch.complex128)
    check(_lib.lib().epb_fourier_phase(_ctx().h, rset.h, ptr(x), nk, ptr(out)))
    return out


def _colstride(t):
    """Column stride (in elements) of a Julia-layout device matrix view; its first axis is contiguous."""
    assert t.stride(-1) == 1, "the first (Julia) axis must be contiguous"
    return t.stride(-2) if t.dim() >= 2 else t.shape[-1]


def fourier_phase_mat(phase, irvec_mat, xkmat):
    """fourier_phase!(phase, irvec_mat, xkmat) with the reference's own operands
    (batched_fourier_core.jl:24-30): irvec_mat the (nr, 3) f64 device matrix of
    _irvec_to_device_matrix (WannierObject.jl:148-152), xkmat (3, nk) f64, phase (nr, nk) c128; column
    views (e.g. P_mk[:, 1:nk]) keep their parent's column stride."""
    nr, three = _jlshape(irvec_mat)
    assert three == 3 and _jlshape(xkmat)[0] == 3
    nk = _jlshape(xkmat)[1]
    assert _jlshape(phase) == (nr, nk)
    check(_lib.lib().epb_fourier_phase_mat(_ctx().h, ptr(irvec_mat), _colstride(irvec_mat), nr, ptr(xkmat),
                                           _colstride(xkmat), nk, ptr(phase), _colstride(phase)))
    return phase


def batched_gemm(transA, transB, A, B, C):
    """batched_gemm!(transA, transB, A, B, C) (src/common/gpu_utils.jl:71-78): C[:, :, b] =
    op(A[:, :, b]) op(B[:, :, b]) for complex128 Julia-layout (rows, cols, batch) device arrays, op 'N',
    'T' or 'C'; strided batch views keep their strides."""
    ra, ca, nb = _jlshape(A)
    rb, cb, nb2 = _jlshape(B)
    m, n, nb3 = _jlshape(C)
    assert nb == nb2 == nb3, "batch sizes differ"
    am, k = (ra, ca) if transA == "N" else (ca, ra)     # op(A) is m x k
    bk, bn = (rb, cb) if transB == "N" else (cb, rb)    # op(B) is k x n
    assert am == m and bn == n and bk == k, "inner or outer dimensions do not match"
    check(_lib.lib().epb_batched_zgemm(_ctx().h, transA.encode(), transB.encode(), m, n, k, ptr(A), _colstride(A),
                                       A.stride(0), ptr(B), _colstride(B), B.stride(0), ptr(C), _colstride(C),
                                       C.stride(0), nb))
    return C


def get_fourier_batched(itp: BatchedWannierInterpolator, xks, out=None, prec=PREC_FP64):
    """out (ndata, nk) = op_r[1:ndata, :] * exp(2 pi i R . x) (batched_interpolator.jl:200-214)."""
    torch = _torch()
    p = itp.parent
    x = _xk_dev(xks)
    nk = x.numel() // 3
    if out is None:
        out = jl_empty((p.ndata, nk), torch.complex128)
    assert _jlshape(out) == (p.ndata, nk)
    ld = p.op_r.shape[1]
    check(_lib.lib().epb_fourier(_ctx().h, ptr(p.op_r), ld, p.ndata, itp.rset.h, ptr(x), nk, ptr(out), prec))
    return out


# ---------------------------------------------------------------------------------------------
def eigvals_batched(Hk, prec=PREC_FP64):
    """E (nw, nk) of a stack (nw, nw, nk); destroys Hk (wannier_to_bloch_batched.jl:30-40)."""
    torch = _torch()
    nw, n2, nk = _jlshape(Hk)
    assert nw == n2
    E = jl_empty((nw, nk), torch.float64)
    check(_lib.lib().epb_eigh_batched(_ctx().h, ptr(Hk), nw, nk, ptr(E), b"N", prec))
    return E


def eigen_batched(Hk, prec=PREC_FP64):
    """(E, U) with U = Hk overwritten (wannier_to_bloch_batched.jl:55-65)."""
    torch = _torch()
    nw, n2, nk = _jlshape(Hk)
    assert nw == n2
    E = jl_empty((nw, nk), torch.float64)
    check(_lib.lib().epb_eigh_batched(_ctx().h, ptr(Hk), nw, nk, ptr(E), b"V", prec))
    return E, Hk


class VarlenBatch:
    """Matrices of uneven order packed back to back (each column-major), as epb_eigh_varlen reads them."""

    def __init__(self, mats, device="cuda"):
        torch = _torch()
        ns = np.array([m.shape[0] for m in mats], dtype=np.int64)
        a_off = np.zeros(len(mats), dtype=np.int64)
        e_off = np.zeros(len(mats), dtype=np.int64)
        if len(mats):
            a_off[1:] = np.cumsum(ns * ns)[:-1]
            e_off[1:] = np.cumsum(ns)[:-1]
        flat = np.concatenate([np.asfortranarray(m, dtype=np.complex128).reshape(-1, order="F") for m in mats]) \
            if len(mats) else np.zeros(1, np.complex128)
        self.ns, self.a_off_h, self.e_off_h = ns, a_off, e_off
        self.A = torch.from_numpy(flat).to(device)
        self.n = torch.from_numpy(ns.astype(np.int32)).to(device)
        self.a_off = torch.from_numpy(a_off).to(device)
        self.e_off = torch.from_numpy(e_off).to(device)
        self.E = torch.empty(max(int(ns.sum()), 1), dtype=torch.float64, device=device)

    def unpack(self):
        """(list of eigenvalue vectors, list of eigenvector matrices) on the host."""
        A = self.A.cpu().numpy()
        E = self.E.cpu().numpy()
        es, us = [], []
        for n, ao, eo in zip(self.ns, self.a_off_h, self.e_off_h):
            es.append(E[eo:eo + n].copy())
            us.append(A[ao:ao + n * n].reshape(n, n, order="F").copy())
        return es, us


def eigen_varlen(mats, prec=PREC_FP64, jobz="V"):
    """Batched eigensolve of matrices of uneven order (upper triangle read, eigenvectors in place);
    returns (eigenvalues, eigenvectors) lists. Replaces eigen_batched over ragged inputs
    (`ext/ElectronPhononCUDAExt.jl:80-115`)."""
    vb = VarlenBatch(mats)
    check(_lib.lib().epb_eigh_varlen(_ctx().h, ptr(vb.A), ptr(vb.a_off), ptr(vb.n), len(mats), ptr(vb.E),
                                     ptr(vb.e_off), jobz.encode(), prec))
    return vb.unpack()


def _fourier_hk_batched(itp, xks, prec=PREC_FP64):
    """H(k) in FP64 in both modes: the mixed mode's FP64 refinement reads H, so an FP64 H(k) gives band
    energies at the FP64 level (the split-BF16 H(k) of the e-ph pass is FP32-level). `prec` is unused."""
    nw = int(round(np.sqrt(itp.parent.ndata)))
    if nw * nw != itp.parent.ndata:
        raise ValueError(f"ndata={itp.parent.ndata} is not a perfect square; expected nw^2 for a Hamiltonian")
    hk = get_fourier_batched(itp, xks, prec=PREC_FP64)
    nk = hk.shape[0]
    return hk.view(nk, nw, nw)


def get_el_eigen_valueonly_batched(itp, xks, prec=PREC_FP64):
    return eigvals_batched(_fourier_hk_batched(itp, xks, prec), prec)


def get_el_eigen_batched(itp, xks, prec=PREC_FP64):
    return eigen_batched(_fourier_hk_batched(itp, xks, prec), prec)


def ph_eigen_batched(itp_dyn, xqs, mass, prec=PREC_FP64):
    """(omega (nm, nq), u (nm, nm, nq)) with device-path semantics (compute_states.jl:285-311)."""
    torch = _torch()
    nm = len(mass)
    dq = get_fourier_batched(itp_dyn, xqs, prec=PREC_FP64)
    nq = dq.shape[0]
    D = dq.view(nq, nm, nm)
    m = torch.as_tensor(np.asarray(mass, dtype=np.float64), device=D.device)
    w = jl_empty((nm, nq), torch.float64)
    check(_lib.lib().epb_ph_eigen_batched(_ctx().h, ptr(D), ptr(m), nm, nq, ptr(w), prec))
    return w, D


# ---------------------------------------------------------------------------------------------
def get_eph_RR_to_kR_batched(ep_ekpR_all, itp_epmat, ks, uks, additional_phase=None, prec=PREC_FP64):
    """(wannier_to_bloch_batched.jl:178-205). ep_ekpR_all: (nw*nband*nm, nr_ep, nk)."""
    epmat = itp_epmat.parent
    nr_ep = epmat.irvec_next.shape[0]
    nw, nband, nk = _jlshape(uks)
    nm = epmat.ndata // (nw * nw * nr_ep)
    assert nm * nw * nw * nr_ep == epmat.ndata
    x = _xk_dev(ks)
    assert x.numel() // 3 == nk
    assert _jlshape(ep_ekpR_all) == (nw * nband * nm, nr_ep, nk)
    if additional_phase is not None:
        assert _jlshape(additional_phase) == (nr_ep, nk)
    check(_lib.lib().epb_eph_RR_to_kR(_ctx().h, ptr(epmat.op_r), nw, nm, nr_ep, itp_epmat.rset.h, ptr(x), nk,
                                      ptr(uks), nband, ptr(additional_phase), ptr(ep_ekpR_all), prec))
    return ep_ekpR_all


def eph_apply_rotations(ep_kq_all, g, ukqs, u_phs, g2_out=None, omega=None):
    """(wannier_to_bloch_batched.jl:442-455). g: (nw, nbk, nm, nq)."""
    nbkq, nbk, nm, nq = _jlshape(ep_kq_all) if ep_kq_all is not None else _jlshape(g2_out)
    nw = _jlshape(ukqs)[0]
    assert _jlshape(g)[:3] == (nw, nbk, nm) and _jlshape(g)[3] == nq
    assert _jlshape(ukqs) == (nw, nbkq, nq)
    assert _jlshape(u_phs) == (nm, nm, nq)
    check(_lib.lib().epb_eph_apply_rotations(_ctx().h, ptr(g), nw * nbk * nm, nw, nbk, nm, nq, ptr(ukqs), nbkq,
                                             ptr(u_phs), ptr(omega), ptr(ep_kq_all), ptr(g2_out)))
    return ep_kq_all


def get_eph_kR_to_kq_batched(ep_kq_all, ep_kR, phase, u_phs, ukqs, g2_out=None, omega=None, prec=PREC_FP64):
    """(wannier_to_bloch_batched.jl:245-273). ep_kR: (nw*nbk*nm, nr_ep), phase: (nr_ep, nq)."""
    nbkq, nbk, nm, nq = _jlshape(ep_kq_all) if ep_kq_all is not None else _jlshape(g2_out)
    nw = _jlshape(ukqs)[0]
    ndata = nw * nbk * nm
    ld, nr_ep = _jlshape(ep_kR)
    assert ld >= ndata
    assert _jlshape(phase) == (nr_ep, nq)
    assert _jlshape(ukqs) == (nw, nbkq, nq)
    assert _jlshape(u_phs) == (nm, nm, nq)
    check(_lib.lib().epb_eph_kR_to_kq(_ctx().h, ptr(ep_kR), ld, nw, nbk, nm, nr_ep, ptr(phase), nq, ptr(ukqs),
                                      nbkq, ptr(u_phs), ptr(omega), ptr(ep_kq_all), ptr(g2_out), prec))
    return ep_kq_all


# ---------------------------------------------------------------------------------------------
# Outer-q loop (the "ph" epmat layout)
def epmat_el_to_ph(epmat_el: WannierObject, nw, nm):
    """The "el"-layout e-ph matrix (rows (i, j, nu, Rp), columns Re) as a "ph"-layout WannierObject
    (rows (i, j, nu, Re), columns Rp, irvec = R_ph, irvec_next = R_el) (src/model_new.jl:551-565)."""
    torch = _torch()
    nr_el = epmat_el.irvec.shape[0]
    nr_ep = epmat_el.irvec_next.shape[0]
    assert epmat_el.ndata == nw * nw * nm * nr_ep
    out = jl_empty((nw * nw * nm * nr_el, nr_ep), torch.complex128, device=epmat_el.op_r.device)
    check(_lib.lib().epb_epmat_el_to_ph(_ctx().h, ptr(epmat_el.op_r), nw, nm, nr_el, nr_ep, ptr(out)))
    obj = WannierObject.__new__(WannierObject)
    obj.irvec, obj.nr, obj.op_r = epmat_el.irvec_next, nr_ep, out
    obj.ndata, obj.irvec_next, obj._id = nw * nw * nm * nr_el, epmat_el.irvec, 0
    obj._irvec_dev = torch.from_numpy(np.ascontiguousarray(obj.irvec)).to(out.device)
    return obj


def get_eph_RR_to_Rq_batched(ep_Rq_all, itp_epmat_ph, xqs, u_phs, prec=PREC_FP64):
    """g(Re, q) in the phonon eigenmode basis for every q of xqs (src/wannier_to_bloch.jl:277-300, a
    list of q at once). itp_epmat_ph: interpolator over the "ph"-layout epmat (its irvec = R_ph);
    u_phs (nm, nm, nq); ep_Rq_all (nw^2 nm, nr_el, nq), rows (i, j, nu). Pass the identity for u_phs to
    keep the Cartesian basis."""
    epmat = itp_epmat_ph.parent
    nr_el = epmat.irvec_next.shape[0]
    nm, _, nq = _jlshape(u_phs)
    nb = epmat.ndata // (nm * nr_el)
    nw = int(round(np.sqrt(nb)))
    assert nw * nw * nm * nr_el == epmat.ndata
    assert _jlshape(u_phs) == (nm, nm, nq)
    assert _jlshape(ep_Rq_all) == (nw * nw * nm, nr_el, nq)
    x = _xk_dev(xqs)
    assert x.numel() // 3 == nq
    check(_lib.lib().epb_eph_RR_to_Rq(_ctx().h, ptr(epmat.op_r), nw, nm, nr_el, itp_epmat_ph.rset.h, ptr(x), nq,
                                      ptr(u_phs), ptr(ep_Rq_all), prec))
    return ep_Rq_all


def get_eph_Rq_to_kq_batched(ep_kq_all, ep_Rq, rset_el, ks, uks, ukqs, g2_out=None, omega=None, prec=PREC_FP64):
    """ep[m, n, nu, k] = sum conj(ukqs[iw, m, k]) g(k, q)[iw, jw, nu] uks[jw, n, k] for one q
    (src/wannier_to_bloch_batched.jl:317-377). ep_Rq: (nw^2 nm, nr_el), one q of
    get_eph_RR_to_Rq_batched; rset_el: R_el as an `_lib.RSet` or an (nr_el, 3) array; optional
    g2_out = |ep|^2 / (2 omega_nu) with omega (nm,)."""
    nbkq, nbk, nm, nk = _jlshape(ep_kq_all) if ep_kq_all is not None else _jlshape(g2_out)
    nw = _jlshape(uks)[0]
    assert _jlshape(uks) == (nw, nbk, nk)
    assert _jlshape(ukqs) == (nw, nbkq, nk)
    rs = rset_el if isinstance(rset_el, _lib.RSet) else _lib.RSet(_ctx(), rset_el)
    assert _jlshape(ep_Rq)[:2] == (nw * nw * nm, rs.nr)
    if g2_out is not None:
        assert omega is not None and omega.numel() >= nm
    x = _xk_dev(ks)
    assert x.numel() // 3 == nk
    check(_lib.lib().epb_eph_Rq_to_kq(_ctx().h, ptr(ep_Rq), nw, nm, rs.h, ptr(x), nk, ptr(uks), nbk, ptr(ukqs),
                                      nbkq, ptr(omega), ptr(ep_kq_all), ptr(g2_out), prec))
    return ep_kq_all


# ---------------------------------------------------------------------------------------------
def window_filter(E, wmin, wmax):
    """Per-k in-window band ranges and the compacted kept-k list (filter.jl:19,40-72).

    Returns (band_min, band_max, keep_idx[:nkeep], nbelow) as device tensors (band indices
    1-based, 0 when empty; keep_idx 0-based ascending).
    """
    torch = _torch()
    nw, nk = _jlshape(E)
    bmin = torch.empty(nk, dtype=torch.int32, device=E.device)
    bmax = torch.empty(nk, dtype=torch.int32, device=E.device)
    keep = torch.empty(max(nk, 1), dtype=torch.int32, device=E.device)
    nkeep = torch.zeros(1, dtype=torch.int64, device=E.device)
    nbelow = torch.empty(nk, dtype=torch.float64, device=E.device)
    check(_lib.lib().epb_window_filter(_ctx().h, ptr(E), nw, nk, float(wmin), float(wmax), ptr(bmin), ptr(bmax),
                                       ptr(keep), ptr(nkeep), ptr(nbelow)))
    n = int(nkeep.item())
    return bmin, bmax, keep[:n], nbelow


def filtered_states(band_min, band_max, nw, capacity=None):
    """FilteredStates of per-k band ranges on the device (band_states.jl:85-121, 283-287).

    Returns (indmap (nw, nk) int64 physical-band map, 0 outside; iks, ibands (n,) int64 1-based;
    n, nband_ignore, nband)."""
    torch = _torch()
    nk = band_min.numel()
    cap = nk * nw if capacity is None else int(capacity)
    indmap = jl_empty((nw, nk), torch.int64)
    iks = torch.empty(max(cap, 1), dtype=torch.int64, device=band_min.device)
    ibands = torch.empty(max(cap, 1), dtype=torch.int64, device=band_min.device)
    counts = torch.zeros(3, dtype=torch.int64, device=band_min.device)
    check(_lib.lib().epb_filtered_states(_ctx().h, ptr(band_min), ptr(band_max), nw, nk, ptr(indmap), ptr(iks),
                                         ptr(ibands), cap, ptr(counts)))
    n, ign, nband = (int(v) for v in counts.cpu())
    return indmap, iks[:min(n, cap)], ibands[:min(n, cap)], n, ign, nband


def fill_iqs(xkq_int, xk_int, ngrid, dense_hash_to_iq):
    """iq (1-based) of x_{k+q} - x_k per column of xkq_int (3, nkq); raises on a miss."""
    torch = _torch()
    nkq = xkq_int.numel() // 3
    iqs = torch.empty(nkq, dtype=torch.int64, device=xkq_int.device)
    xk = np.ascontiguousarray(np.asarray(xk_int, dtype=np.int64))
    check(_lib.lib().epb_fill_iqs(_ctx().h, ptr(xkq_int), nkq, xk.ctypes.data, int(ngrid[0]), int(ngrid[1]),
                                  int(ngrid[2]), ptr(dense_hash_to_iq), ptr(iqs)))
    return iqs


# ---------------------------------------------------------------------------------------------
def eph_window_scatter(g2_out, omega_out, g2vals, imap_i_col, imap_f, ikqs, omega, ni_stride, i0):
    """eph_window_scatter! (src/calculator/calculator_utils.jl:36-50): device arrays in Julia layout,
    index maps int64 1-based (0 = out of window)."""
    nbkq, nbk, nm, nqb = _jlshape(g2vals)
    ld_f = _jlshape(imap_f)[0]
    check(_lib.lib().epb_eph_window_scatter(_ctx().h, ptr(g2_out), ptr(omega_out), ptr(g2vals), ptr(imap_i_col),
                                            ptr(imap_f), ld_f, ptr(ikqs), ptr(omega), nbkq, nbk, nm, nqb,
                                            int(ni_stride), int(i0)))


def bte_window_accumulate(sout, sin, g2vals, omega, imap_i_at_k, imap_f, ikqs, e_i, e_f, wf, mus, ts, etas, method,
                          omega_cutoff, i0):
    """bte_window_accumulate! (src/boltzmann/boltzmann_calculator.jl:336-362). sout (n_i, nT),
    sin (ni_tile, n_f, nT) or None, Julia layout device arrays."""
    nbkq, nbk, nm, nqb = _jlshape(g2vals)
    n_i, nT = _jlshape(sout)
    ni_tile, n_f = (_jlshape(sin)[:2] if sin is not None else (0, 0))
    ld_f = _jlshape(imap_f)[0]
    check(_lib.lib().epb_bte_window_accumulate(_ctx().h, ptr(sout), n_i, ptr(sin), ni_tile, n_f, ptr(g2vals), ptr(omega),
                                               ptr(imap_i_at_k), ptr(imap_f), ld_f, ptr(ikqs), ptr(e_i), ptr(e_f),
                                               ptr(wf), ptr(mus), ptr(ts), ptr(etas), nT, int(method),
                                               float(omega_cutoff), nbkq, nbk, nm, nqb, int(i0)))
