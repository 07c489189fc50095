"""CPU FP64 oracle for the Wannier->Bloch electron-phonon hot path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only `tests/`, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of `bench.py` may import it. It restates, in numpy/scipy,
the algorithm of jaemolihm/ElectronPhonon.jl for the functions on the hot path; each function cites
the reference file:line it follows (paths relative to the reference project root).

Pinning. The reference is Julia and cannot run in this environment (no Julia toolchain), so no
output of the reference itself is available. The restatement is pinned instead to the reference's
own known-answer and identity tests (`tests/test_oracle.py` reproduces each):
  * `test/test_gpu.jl:127-144`  phase vs scalar cispi, max error <= 4 eps;
  * `test/test_gpu.jl:44-122`   list-batched drivers == per-k/per-q functions, rtol 1e-10;
  * `test/test_gpu.jl:156-211`  k+q convention identity, rtol 1e-13, bit-identical phase method;
  * `test/test_gpu.jl:260-273`  eigen reconstruction U diag(E) U^dagger == H, eigenvalues vs LAPACK;
  * `test/test_diagonalize.jl:18-48` electron/phonon eigen identities;
  * `test/test_iq_build.jl:230-310` integer iq hash == xk_to_ik;
  * `test/boltzmann/test_gpu_boltzmann_calculator.jl:5-29` golden BTE increments (rtol 1e-12).
The eigensolver is LAPACK ZHEEV (scipy `eigh(driver="ev")`), the routine of
`src/common/AllocatedLAPACK.jl:72-102`.

Array conventions: a Julia column-major array of size (n1, n2, ...) is a numpy array of the same
shape in Fortran order; indices are 0-based here, 1-based in the reference.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg

# src/common/units.jl:25-26 and src/common/constants.jl:5-6
UNIT_EV = 0.03674932248 * 2
UNIT_MEV = 0.03674932248 * 2 * 1e-3
UNIT_K = 3.166810508e-6 * 2
OMEGA_ACOUSTIC = 0.01 * UNIT_MEV
ELECTRON_DEGEN_CUTOFF = 0.01 * UNIT_MEV


# --------------------------------------------------------------------------------------------
# Fourier transform (L3)

def cispi(x):
    """Julia `cispi(x)` = exp(i pi x) with exact argument reduction (reduce x mod 2 first)."""
    x = np.asarray(x, dtype=np.float64)
    r = x - 2.0 * np.rint(x * 0.5)          # exact for |x| < 2^52; r in [-1, 1]
    return np.cos(np.pi * r) + 1j * np.sin(np.pi * r)


def fourier_phase(irvec, xk):
    """phase[ir, j] = cispi(2 (R_ir . x_j)); `src/wannier/batched_fourier_core.jl:24-30`.

    irvec: (nr, 3) integers; xk: (3, nk). Dot product evaluated as (R1 x1 + R2 x2) + R3 x3.
    """
    r = np.asarray(irvec, dtype=np.float64)
    x = np.asarray(xk, dtype=np.float64)
    t = r[:, 0:1] * x[0:1, :] + r[:, 1:2] * x[1:2, :] + r[:, 2:3] * x[2:3, :]
    return cispi(2.0 * t)


def fourier_batched(op_r, ndata, irvec, xk):
    """out = op_r[0:ndata, :] @ phase; `src/wannier/batched_fourier_core.jl:117-139`."""
    return np.asfortranarray(op_r[:ndata, :] @ fourier_phase(irvec, xk))


def get_fourier(op_r, ndata, irvec, xk1):
    """Per-k 'normal' Fourier (GEMV); `src/wannier/WannierInterpolator.jl:121-139`."""
    return op_r[:ndata, :] @ fourier_phase(irvec, np.asarray(xk1).reshape(3, 1))[:, 0]


# --------------------------------------------------------------------------------------------
# Eigensolvers

def _zheev(a, jobz):
    """LAPACK ZHEEV on the upper triangle (`src/common/AllocatedLAPACK.jl:82-102`)."""
    if jobz == "N":
        return scipy.linalg.eigh(a, lower=False, eigvals_only=True, driver="ev"), None
    w, v = scipy.linalg.eigh(a, lower=False, driver="ev")
    return w, v


def eigvals_batched(hk):
    """(nw, nw, nk) -> E (nw, nk); `src/wannier_to_bloch_batched.jl:30-40`."""
    nw, _, nk = hk.shape
    e = np.empty((nw, nk), order="F")
    for ik in range(nk):
        e[:, ik] = _zheev(hk[:, :, ik], "N")[0]
    return e


def eigen_batched(hk):
    """(nw, nw, nk) -> (E, U); no gauge fix; `src/wannier_to_bloch_batched.jl:55-65`."""
    nw, _, nk = hk.shape
    e = np.empty((nw, nk), order="F")
    u = np.empty_like(hk, order="F")
    for ik in range(nk):
        w, v = _zheev(hk[:, :, ik], "V")
        e[:, ik] = w
        u[:, :, ik] = v
    return e, u


def degeneracy_perturbation_matrix(n):
    """EPW perturbation P[j,i] = (0.25644832 + 0.005(i+j)) + i 0.0125 (j-i), 1-based i, j;
    `src/diagonalize.jl:11-18`."""
    i = np.arange(1, n + 1)[None, :]
    j = np.arange(1, n + 1)[:, None]
    return (0.25644832 + 0.005 * (i + j)) + 1j * (0.0125 * (j - i))


def solve_eigen_el(hk):
    """Per-k eigen with the EPW degenerate-gauge fix; `src/diagonalize.jl:35-86`."""
    e, u = _zheev(np.array(hk), "V")
    n = hk.shape[0]
    if not np.any(np.abs(np.diff(e)) < ELECTRON_DEGEN_CUTOFF):
        return e, u
    p = degeneracy_perturbation_matrix(n)
    degen_e = e[0]
    degen_from = 0
    for i in range(n - 1):
        if abs(degen_e - e[i + 1]) > ELECTRON_DEGEN_CUTOFF:
            degen_to = i
        elif i == n - 2:
            degen_to = i + 1
        else:
            continue
        if degen_to - degen_from + 1 > 1:
            rng = slice(degen_from, degen_to + 1)
            pm = u[:, rng].conj().T @ p @ u[:, rng]
            _, pv = _zheev(pm, "V")
            u[:, rng] = u[:, rng] @ pv
        degen_e = e[i + 1]
        degen_from = i + 1
    return e, u


def solve_eigen_ph(dynq, mass):
    """omega = sign(l) sqrt|l|, u[i,:] /= sqrt(m_i); `src/diagonalize.jl:104-127`."""
    e, u = _zheev(np.array(dynq), "V")
    w = np.where(e >= 0, np.sqrt(np.abs(e)), -np.sqrt(np.abs(e)))
    u = u / np.sqrt(np.asarray(mass))[:, None]
    return w, u


def get_ph_eigen(xq, dyn_op_r, irvec_ph, mass):
    """D(q)/sqrt(m_i m_j) -> eigen; `src/wannier_to_bloch.jl:186-205` (non-polar)."""
    nm = len(mass)
    d = get_fourier(dyn_op_r, nm * nm, irvec_ph, xq).reshape(nm, nm, order="F")
    sm = np.sqrt(np.asarray(mass))
    d = d / sm[:, None] / sm[None, :]
    return solve_eigen_ph(d, mass)


def ph_eigen_batched(xqs, dyn_op_r, irvec_ph, mass):
    """Phonons over a q list, device-path semantics (`src/compute_states.jl:285-311`): no gauge fix."""
    nm = len(mass)
    dq = fourier_batched(dyn_op_r, nm * nm, irvec_ph, xqs).reshape(nm, nm, -1, order="F")
    sm = np.sqrt(np.asarray(mass))
    dq = dq / sm[:, None, None] / sm[None, :, None]
    nq = dq.shape[2]
    w = np.empty((nm, nq), order="F")
    u = np.empty((nm, nm, nq), dtype=np.complex128, order="F")
    for iq in range(nq):
        w[:, iq], u[:, :, iq] = solve_eigen_ph(dq[:, :, iq], mass)
    return w, u


# --------------------------------------------------------------------------------------------
# Electron-phonon chain

def get_eph_RR_to_kR(epmat_op_r, irvec_el, nr_ep, nw, nmodes, xk1, uk):
    """Per-k RR->kR: g(k,Rp) rotated on the k (jw) leg by uk; `src/wannier_to_bloch.jl:365-393`.
    Returns (nw*nband*nmodes, nr_ep)."""
    nband = uk.shape[1]
    gk = get_fourier(epmat_op_r, epmat_op_r.shape[0], irvec_el, xk1)
    gk = gk.reshape(nw, nw, nmodes, nr_ep, order="F")
    out = np.empty((nw, nband, nmodes, nr_ep), dtype=np.complex128, order="F")
    for ir in range(nr_ep):
        for im in range(nmodes):
            out[:, :, im, ir] = gk[:, :, im, ir] @ uk
    return out.reshape(nw * nband * nmodes, nr_ep, order="F")


def get_eph_RR_to_kR_batched(epmat_op_r, irvec_el, nr_ep, nw, nmodes, xks, uks, additional_phase=None):
    """Batched RR->kR (`src/wannier_to_bloch_batched.jl:178-205`):
    out[iw, n, (nu,p), k] = sum_jw g[iw, jw, (nu,p), k] uk[jw, n, k] (* additional_phase[p, k])."""
    nk = xks.shape[1]
    nband = uks.shape[1]
    m = nmodes * nr_ep
    g = fourier_batched(epmat_op_r, epmat_op_r.shape[0], irvec_el, xks)
    g4 = g.reshape(nw, nw, m, nk, order="F")
    out = np.einsum("ijmk,jnk->inmk", g4, uks)
    out = out.reshape(nw * nband * nmodes, nr_ep, nk, order="F")
    if additional_phase is not None:
        out = out * np.asarray(additional_phase).reshape(1, nr_ep, nk)
    return np.asfortranarray(out)


def eph_apply_rotations(g, ukqs, u_phs, omega=None):
    """ep = ukq^dagger g u_ph per q, and g2 = |ep|^2/(2 omega)
    (`src/wannier_to_bloch_batched.jl:442-455`). g: (nw, nbk, nm, nq)."""
    tmp = np.einsum("imq,inaq->mnaq", ukqs.conj(), g)
    ep = np.asfortranarray(np.einsum("mnaq,abq->mnbq", tmp, u_phs))
    g2 = None
    if omega is not None:
        g2 = np.asfortranarray(np.abs(ep) ** 2 / (2.0 * np.asarray(omega)[None, None, :, :]))
    return ep, g2


def get_eph_kR_to_kq_batched(ep_kR, phase, u_phs, ukqs, nbk, omega=None):
    """Batched kR->kq for one k (`src/wannier_to_bloch_batched.jl:245-273`).
    ep_kR: (nw*nbk*nm, nr_ep); phase: (nr_ep, nq)."""
    nw = ukqs.shape[0]
    nm = u_phs.shape[0]
    nq = phase.shape[1]
    g = (ep_kR @ phase).reshape(nw, nbk, nm, nq, order="F")
    return eph_apply_rotations(g, ukqs, u_phs, omega)


def get_eph_kR_to_kq(ep_kR, irvec_ep, xq1, u_ph, ukq, nbk):
    """Per-q kR->kq (`src/wannier_to_bloch.jl:409-443`): ep = ukq^dagger g(k,q) u_ph."""
    nw = ukq.shape[0]
    nm = u_ph.shape[0]
    g = get_fourier(ep_kR, ep_kR.shape[0], irvec_ep, xq1).reshape(nw, nbk * nm, order="F")
    ab1 = (ukq.conj().T @ g).reshape(-1, nm, order="F")
    return (ab1 @ u_ph).reshape(ukq.shape[1], nbk, nm, order="F")


def epmat_el_to_ph(op_r_el, nw, nmodes, nr_el, nr_ep):
    """(i, j, nu, Rp, Re) -> (i, j, nu, Re, Rp), the two layouts of `src/model_new.jl:551-565`
    (permutedims [1,2,3,5,4], `src/model.jl:80-81,293-296`)."""
    a = np.asarray(op_r_el).reshape(nw * nw * nmodes, nr_ep, nr_el, order="F")
    return np.asfortranarray(a.transpose(0, 2, 1).reshape(nw * nw * nmodes * nr_el, nr_ep, order="F"))


def get_eph_RR_to_Rq(op_r_ph, irvec_ep, nw, nmodes, nr_el, xq1, u_ph):
    """g(Re, q) rotated into the phonon eigenmode basis, one Re at a time
    (`src/wannier_to_bloch.jl:277-300`). Returns (nw*nw*nmodes, nr_el), rows (i, j, nu)."""
    g = get_fourier(op_r_ph, op_r_ph.shape[0], irvec_ep, xq1).reshape(nw * nw, nmodes, nr_el, order="F")
    out = np.empty_like(g)
    for ir in range(nr_el):
        out[:, :, ir] = g[:, :, ir] @ u_ph
    return out.reshape(nw * nw * nmodes, nr_el, order="F")


def get_eph_Rq_to_kq_batched(g_Rq, irvec_el, xks, uks, ukqs, nmodes):
    """ep[m, n, nu, k] = sum_{iw, jw} conj(ukqs[iw, m, k]) g(k, q)[iw, jw, nu] uks[jw, n, k]
    (`src/wannier_to_bloch_batched.jl:317-377`; the per-k form `src/wannier_to_bloch.jl:326-350`)."""
    nw = uks.shape[0]
    nk = xks.shape[1]
    g = fourier_batched(g_Rq, g_Rq.shape[0], irvec_el, xks).reshape(nw, nw, nmodes, nk, order="F")
    return np.asfortranarray(np.einsum("imk,ijak,jnk->mnak", ukqs.conj(), g, uks))


def outer_q_record(model, xks, xqs, wtk=None, window_k=(-np.inf, np.inf), window_kq=(-np.inf, np.inf),
                   phonon_basis="eigenmode"):
    """A[iq] = sum_k wtk[k] sum_{m in window_kq(k+q), n in window_k(k), nu} |ep[m, n, nu]|^2 through the
    per-point outer-q chain (`src/wannier_to_bloch.jl:277-350`); k with an empty window_k range are
    dropped (`src/filter.jl:40-72`). The record calculator of test/test_gpu.jl:589-654."""
    nw, nm = model.nw, model.nmodes
    ham, ep = model.el_ham, model.epmat
    nr_el, nr_ep = ep.irvec.shape[0], ep.irvec_next.shape[0]
    op_ph = epmat_el_to_ph(ep.op_r, nw, nm, nr_el, nr_ep)
    xks = np.asarray(xks, dtype=np.float64).reshape(3, -1)
    xqs = np.asarray(xqs, dtype=np.float64).reshape(3, -1)
    nk, nq = xks.shape[1], xqs.shape[1]
    w = np.ones(nk) if wtk is None else np.asarray(wtk, dtype=np.float64)
    hk = fourier_batched(ham.op_r, ham.ndata, ham.irvec, xks).reshape(nw, nw, nk, order="F")
    Ek, Uk = eigen_batched(hk)
    A = np.zeros(nq)
    for iq in range(nq):
        xq = xqs[:, iq]
        if phonon_basis == "eigenmode":
            _, u = ph_eigen_batched(xq.reshape(3, 1), model.ph_dyn.op_r, model.ph_dyn.irvec, model.mass)
            uph = u[:, :, 0]
        else:
            uph = np.eye(nm, dtype=np.complex128)
        gRq = get_eph_RR_to_Rq(op_ph, ep.irvec_next, nw, nm, nr_el, xq, uph)
        xkq = xks + xq[:, None]
        hkq = fourier_batched(ham.op_r, ham.ndata, ham.irvec, xkq).reshape(nw, nw, nk, order="F")
        Ekq, Ukq = eigen_batched(hkq)
        for k in range(nk):
            s, t = inside_window(Ek[:, k], *window_k)
            if t < s:
                continue
            s2, t2 = inside_window(Ekq[:, k], *window_kq)
            if t2 < s2:
                continue
            e = get_eph_Rq_to_kq_batched(gRq, ep.irvec, xks[:, k:k + 1], Uk[:, s - 1:t, k:k + 1],
                                         Ukq[:, s2 - 1:t2, k:k + 1], nm)
            A[iq] += w[k] * float(np.sum(np.abs(e) ** 2))
    return A


def epstate_set_g2(ep, omega):
    """g2[:,:,nu] = |ep|^2 / (2 omega_nu), no frequency floor; `src/EPState.jl:73-81`."""
    return np.abs(ep) ** 2 * (1.0 / (2.0 * np.asarray(omega)))[None, None, :]


# --------------------------------------------------------------------------------------------
# Energy window / filtering

def inside_window(e, wmin, wmax):
    """searchsortedfirst(e,wmin):searchsortedlast(e,wmax) as a 1-based (start, stop) pair;
    `src/filter.jl:19`. Empty when stop < start."""
    e = np.asarray(e)
    start = int(np.searchsorted(e, wmin, side="left")) + 1
    stop = int(np.searchsorted(e, wmax, side="right"))
    return start, stop


def filter_kpoints(e, weights, wmin, wmax):
    """`_filter_kpoints` device branch semantics (`src/filter.jl:40-100`) on given eigenvalues.
    Returns ik_keep (bool), band_min_per_k, band_max_per_k (1-based, 0 if none),
    nelec_below_window (sum of (start-1)*w), band_min, band_max."""
    nw, nk = e.shape
    keep = np.zeros(nk, dtype=bool)
    bmin = np.zeros(nk, dtype=np.int64)
    bmax = np.zeros(nk, dtype=np.int64)
    nbelow = np.zeros(nk)
    for ik in range(nk):
        s, t = inside_window(e[:, ik], wmin, wmax)
        nbelow[ik] = (s - 1) * weights[ik]
        if t >= s:
            keep[ik] = True
            bmin[ik], bmax[ik] = s, t
    return dict(ik_keep=keep, band_min_per_k=bmin, band_max_per_k=bmax,
                nelec_below_window=float(nbelow.sum()),
                band_min=int(bmin.min()) if nk else 0, band_max=int(bmax.max()) if nk else 0)


def filtered_states_indmap(ik_keep, bmin, bmax):
    """(k, band) -> 1-based state index, 0 = outside (`src/band_states.jl:99-121`), states ordered
    by k then band. Returns (iks, ibands, indmap[nband, nk], nband_ignore)."""
    iks, ibs = [], []
    for ik in np.nonzero(ik_keep)[0]:
        for b in range(bmin[ik], bmax[ik] + 1):
            iks.append(ik + 1)
            ibs.append(b)
    iks = np.asarray(iks, dtype=np.int64)
    ibs = np.asarray(ibs, dtype=np.int64)
    nk = len(ik_keep)
    if len(ibs) == 0:
        return iks, ibs, np.zeros((0, nk), dtype=np.int64), 0
    ign = int(ibs.min()) - 1
    nband = int(ibs.max()) - ign
    indmap = np.zeros((nband, nk), dtype=np.int64, order="F")
    for i, (k, b) in enumerate(zip(iks, ibs)):
        indmap[b - ign - 1, k - 1] = i + 1
    return iks, ibs, indmap, ign


# --------------------------------------------------------------------------------------------
# Grid hash (`src/common/kpoints.jl:614-650`, `src/calculator/run_eph_over_k_and_kq.jl:565-582`)

def grid_coords_reduced(xk, ngrid, shift):
    """mod(round(Int, (xk - shift) * ngrid), ngrid) per axis (Julia round = ties to even)."""
    xk = np.asarray(xk, dtype=np.float64)
    c = np.rint((xk - np.asarray(shift, dtype=np.float64)) * np.asarray(ngrid))
    return np.mod(c.astype(np.int64), np.asarray(ngrid, dtype=np.int64))


def wrap_reduced(d, ng):
    if not (-ng < d < 2 * ng):
        raise ValueError(f"wrap_reduced({d}, {ng}) outside (-ng, 2ng)")
    return d + ng if d < 0 else (d - ng if d >= ng else d)


def hash_xk(xk, ngrid, shift):
    c = grid_coords_reduced(xk, ngrid, shift)
    return int((c[0] * ngrid[1] + c[1]) * ngrid[2] + c[2])


def fill_iqs(q_dense_hash_to_iq, ngrid, xkqs_int, xk_int):
    """iq (1-based) of x_{k+q} - x_k for each k+q of a tile; raises on a miss."""
    out = np.empty(xkqs_int.shape[1], dtype=np.int64)
    for j in range(xkqs_int.shape[1]):
        h = [wrap_reduced(int(xkqs_int[d, j] - xk_int[d]), ngrid[d]) for d in range(3)]
        hsh = (h[0] * ngrid[1] + h[1]) * ngrid[2] + h[2]
        iq = int(q_dense_hash_to_iq[hsh])
        if iq < 1:
            raise ValueError("kq - k = q point not found in precomputed qpts")
        out[j] = iq
    return out


# --------------------------------------------------------------------------------------------
# BTE scattering increments (`src/boltzmann/bte_scattering_core.jl:9-84`, `src/common/smearing.jl:29-57`)

def smearing_gaussian(de, eta):
    return (1.0 / math.sqrt(math.pi)) / eta * math.exp(-(de / eta) ** 2)


def _occ_fd(e, t):
    return 1.0 / (math.exp(e / t) + 1.0)


def _occ_fd_deriv(e, t):
    return -1.0 / (2.0 + math.exp(e / t) + math.exp(-e / t)) / t


def _occ_boson(e, t):
    return 0.0 if e == 0 else 1.0 / math.expm1(e / t)


def bte_scattering_increments(method, ek, ekq, wq, g2, wtq, mu, temp, eta):
    """(s_out, s_in) for one (k, k+q, mode) triple; Gaussian smearing of width eta."""
    d1 = smearing_gaussian(ek - ekq + wq, eta)
    d2 = smearing_gaussian(ek - ekq - wq, eta)
    if d1 == 0.0 and d2 == 0.0:
        return 0.0, 0.0
    nq = _occ_boson(wq, temp)
    fk = _occ_fd(ek - mu, temp)
    fkq = _occ_fd(ekq - mu, temp)
    if method == 1:
        f1o, f2o = nq + fkq, nq + 1 - fkq
        f1i, f2i = nq + fk, nq + 1 - fk
    elif method == 2:
        preo = fkq * (1 - fkq) / (fk * (1 - fk))
        f1o, f2o = preo * (nq + 1 - fk), preo * (nq + fk)
        prei = fk * (1 - fk) / (fkq * (1 - fkq))
        f1i, f2i = prei * (nq + 1 - fkq), prei * (nq + fkq)
    elif method == 3:
        preo = (1 - fkq) / (1 - fk)
        f1o, f2o = preo * nq, preo * (nq + 1)
        prei = (1 - fk) / (1 - fkq)
        f1i, f2i = prei * nq, prei * (nq + 1)
    elif method == 4:
        preo = fkq / fk
        f1o, f2o = preo * (nq + 1), preo * nq
        prei = fk / fkq
        f1i, f2i = prei * (nq + 1), prei * nq
    elif method == 5:
        dfk = _occ_fd_deriv(ek - mu, temp)
        dfkq = _occ_fd_deriv(ekq - mu, temp)
        f1o = math.sqrt(nq * (nq + 1) * dfkq / dfk)
        f2o = f1o
        f1i = math.sqrt(nq * (nq + 1) * dfk / dfkq)
        f2i = f1i
    else:
        ndo = _occ_boson(ekq - ek, temp)
        f1o, f2o = ndo + fkq, -(ndo + fkq)
        ndi = _occ_boson(ek - ekq, temp)
        f1i, f2i = ndi + fk, -(ndi + fk)
    pref = 2 * math.pi * wtq * g2
    so = ((0.0 if d1 == 0 else d1 * f1o) + (0.0 if d2 == 0 else d2 * f2o)) * pref
    si = ((0.0 if d2 == 0 else d2 * f1i) + (0.0 if d1 == 0 else d1 * f2i)) * pref
    return so, si


# --------------------------------------------------------------------------------------------
# Whole e-ph pass for explicit (k, q) pairs (semantics of `run_eph_over_k_and_q`,
# `src/calculator/run_eph_over_k_and_q.jl:251-330`, non-polar, no energy conservation)

def eph_pairs(model, xks, xqs, pairs, window=(-np.inf, np.inf), gauge_fix=False):
    """|g|^2 for each (ik, iq) pair in `pairs`, in the q convention.

    Returns a list of dicts with ek, ekq (full), rng_k, rng_kq (1-based inclusive band windows),
    omega (nm), g2 (nbkq, nbk, nm) for kept pairs (None when a window is empty), plus ep.
    The electron eigensolve is the batched one (no gauge fix) unless `gauge_fix`.
    """
    ham = model.el_ham
    ep = model.epmat
    nw, nm = model.nw, model.nmodes
    nr_ep = ep.irvec_next.shape[0]
    res = []
    cache_k = {}
    for ik, iq in pairs:
        xk = xks[:, ik]
        xq = xqs[:, iq]
        if ik not in cache_k:
            hk = get_fourier(ham.op_r, ham.ndata, ham.irvec, xk).reshape(nw, nw, order="F")
            ek, uk = solve_eigen_el(hk) if gauge_fix else _zheev(hk, "V")
            s, t = inside_window(ek, *window)
            if t >= s:
                ukw = uk[:, s - 1:t]
                kR = get_eph_RR_to_kR(ep.op_r, ep.irvec, nr_ep, nw, nm, xk, ukw)
            else:
                kR = None
            cache_k[ik] = (ek, uk, (s, t), kR)
        ek, uk, (s, t), kR = cache_k[ik]
        xkq = xk + xq
        hkq = get_fourier(ham.op_r, ham.ndata, ham.irvec, xkq).reshape(nw, nw, order="F")
        ekq, ukq = solve_eigen_el(hkq) if gauge_fix else _zheev(hkq, "V")
        s2, t2 = inside_window(ekq, *window)
        w, uph = get_ph_eigen(xq, model.ph_dyn.op_r, model.ph_dyn.irvec, model.mass)
        entry = dict(ik=ik, iq=iq, ek=ek, ekq=ekq, rng_k=(s, t), rng_kq=(s2, t2), omega=w,
                     g2=None, ep=None)
        if kR is not None and t2 >= s2:
            nbk = t - s + 1
            e = get_eph_kR_to_kq(kR, ep.irvec_next, xq, uph, ukq[:, s2 - 1:t2], nbk)
            entry["ep"] = e
            entry["g2"] = epstate_set_g2(e, w)
        res.append(entry)
    return res


# --------------------------------------------------------------------------------------------
# Calculator hooks of the batched loop

def eph_window_scatter(g2_out, om_out, g2vals, imap_i_col, imap_f, ikqs, om, ni_stride, i0):
    """`src/calculator/calculator_utils.jl:36-50` on flat 0-based numpy outputs (1-based maps)."""
    nbkq, nbk, nm, nqb = g2vals.shape
    for j in range(nqb):
        for nu in range(nm):
            for n in range(nbk):
                for m in range(nbkq):
                    i = imap_i_col[n]
                    f = imap_f[m, ikqs[j] - 1]
                    if i > 0 and f > 0:
                        lin = nu + nm * (i - i0 - 1) + nm * ni_stride * (f - 1)
                        g2_out[lin] = g2vals[m, n, nu, j]
                        om_out[lin] = om[nu, j]


def ind_range_for_k_range(iks, kstart, kend):
    """1-based states with kstart <= iks[i] <= kend as a range; ValueError when they are not contiguous
    (`src/band_states.jl:416-428`)."""
    idx = [i + 1 for i, k in enumerate(iks) if kstart <= k <= kend]
    if not idx:
        return range(1, 1)
    if idx[-1] - idx[0] + 1 != len(idx):
        raise ValueError("non-contiguous state range")
    return range(idx[0], idx[-1] + 1)


def tile_capacity(iks, nk, n_batch_max):
    """ni_cap of `tile_begin!` (`src/calculator/tiled_device_output.jl:107-108`)."""
    return max((len(ind_range_for_k_range(iks, ks, min(ks + n_batch_max - 1, nk))) for ks in range(1, nk + 1, n_batch_max)),
               default=0)


def bte_window_accumulate(sout, sin, g2vals, om, imap_i_at_k, imap_f, ikqs, e_i, e_f, wf, mus, ts, etas, method,
                          omega_cutoff, i0):
    """`src/boltzmann/boltzmann_calculator.jl:336-362` (1-based maps, 0-based numpy arrays)."""
    nbkq, nbk, nm, nqb = g2vals.shape
    for j in range(nqb):
        for n in range(nbk):
            for m in range(nbkq):
                i = imap_i_at_k[n]
                if i <= 0:
                    continue
                f = imap_f[m, ikqs[j] - 1]
                if f <= 0:
                    continue
                for iT in range(len(mus)):
                    so = si = 0.0
                    for nu in range(nm):
                        if om[nu, j] < omega_cutoff:
                            continue
                        a, b = bte_scattering_increments(method, e_i[i - 1], e_f[f - 1], om[nu, j], g2vals[m, n, nu, j],
                                                         wf[f - 1], mus[iT], ts[iT], etas[iT])
                        so += a
                        si += b
                    sout[i - 1, iT] += so
                    if sin is not None:
                        sin[i - i0 - 1, f - 1, iT] = si
