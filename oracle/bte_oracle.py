"""CPU FP64 oracle of the SERTA Boltzmann consumer (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only `tests/`, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of `bench.py` may import it.

It restates, for commensurate k = q grids, the reference's batched k / k+q loop feeding the
Boltzmann calculator, on the functions of `epb_oracle` (each pinned by `tests/test_oracle.py`):
  * electron states on the grid: H(k) Fourier sum + ZHEEV, energy window per k (`src/filter.jl:19`);
  * band velocities v_n(k) = Re <u_n| dH/dk |u_n>, dH/dk_a = sum_R i R_cart,a H(R) e^{2 pi i x.R}
    (the diagonal velocity of `src/electron_state.jl:130-150` / the `vdiag` of the batched path);
  * phonons on the q grid (`src/diagonalize.jl:104-127`), omega_cutoff skip
    (`src/boltzmann/boltzmann_calculator.jl:355-357`);
  * |g|^2 of every in-window (n at k, m at k+q, nu) triple in the q convention
    (`src/wannier_to_bloch.jl:365-443`, `src/EPState.jl:73-81`);
  * out-scattering rates S_out[i] = sum_{f, nu} increments of `bte_scattering_increments`
    (`src/boltzmann/bte_scattering_core.jl:9-84`), weight 1/nq per final state
    (`src/boltzmann/boltzmann_calculator.jl:336-362`);
  * SERTA conductivity sigma = (spin / V) sum_i w_k (-f'(e_i - mu) / S_out[i]) v_i v_i^T
    (`src/boltzmann/electron_lbte.jl:43-49,153-185`).
Grid order: k fastest (`src/common/kpoints.jl:135-153`): ik = (i1 ng + i2) ng + i3.
"""
from __future__ import annotations

import math

import numpy as np

from . import epb_oracle as O


def grid_points(ng):
    ik = np.arange(ng ** 3)
    c = np.stack([ik // (ng * ng), (ik // ng) % ng, ik % ng])
    return np.asfortranarray(c / ng), c


def velocities(op_r, nw, irvec, lattice, x, U):
    """v[a, n, k] = Re(u_n^H dH_a u_n) for the eigenvectors U (nw, nw, nk) at points x (3, nk)."""
    rc = np.asarray(lattice, dtype=np.float64) @ np.asarray(irvec, dtype=np.float64).T  # (3, nr) Cartesian
    ph = O.fourier_phase(irvec, x)  # (nr, nk)
    v = np.zeros((3, nw, x.shape[1]))
    for a in range(3):
        dop = op_r[: nw * nw, :] * (1j * rc[a])[None, :]
        dh = (dop @ ph).reshape(nw, nw, -1, order="F")
        for k in range(x.shape[1]):
            u = U[:, :, k]
            v[a, :, k] = np.real(np.einsum("in,ij,jn->n", u.conj(), dh[:, :, k], u))
    return v


def serta(model, ng, wmin, wmax, mu, temp, eta, method=5, omega_cutoff=O.OMEGA_ACOUSTIC, lattice=np.eye(3),
          volume=1.0, spin=2.0):
    """SERTA conductivity (3, 3) and per-state inverse lifetimes on an ng^3 k = q grid."""
    nw, nm = model.nw, model.nmodes
    ham, ep = model.el_ham, model.epmat
    nr_ep = ep.irvec_next.shape[0]
    x, c = grid_points(ng)
    N = x.shape[1]
    hk = O.fourier_batched(ham.op_r, nw * nw, ham.irvec, x).reshape(nw, nw, N, order="F")
    E, U = O.eigen_batched(np.asfortranarray(hk))
    win = [O.inside_window(E[:, k], wmin, wmax) for k in range(N)]
    w_ph, u_ph = O.ph_eigen_batched(x, model.ph_dyn.op_r, model.ph_dyn.irvec, model.mass)
    kept = [k for k in range(N) if win[k][1] >= win[k][0]]
    V = velocities(ham.op_r, nw, ham.irvec, lattice, x[:, kept], U[:, :, kept]) if kept else None
    sout = {}
    npairs = 0
    for kk, k in enumerate(kept):
        s, t = win[k]
        kR = O.get_eph_RR_to_kR(ep.op_r, ep.irvec, nr_ep, nw, nm, x[:, k], U[:, s - 1:t, k])
        for iq in range(N):
            ikq = int((((c[0, k] + c[0, iq]) % ng) * ng + (c[1, k] + c[1, iq]) % ng) * ng + (c[2, k] + c[2, iq]) % ng)
            s2, t2 = win[ikq]
            if t2 < s2:
                continue
            npairs += 1
            e = O.get_eph_kR_to_kq(kR, ep.irvec_next, x[:, iq], u_ph[:, :, iq], U[:, s2 - 1:t2, ikq], t - s + 1)
            g2 = O.epstate_set_g2(e, w_ph[:, iq])  # (nbkq, nbk, nm)
            for n in range(t - s + 1):
                acc = 0.0
                for m in range(t2 - s2 + 1):
                    for nu in range(nm):
                        if w_ph[nu, iq] < omega_cutoff:
                            continue
                        so, _ = O.bte_scattering_increments(method, E[s - 1 + n, k], E[s2 - 1 + m, ikq], w_ph[nu, iq],
                                                            g2[m, n, nu], 1.0 / N, mu, temp, eta)
                        acc += so
                sout[(k, s - 1 + n)] = sout.get((k, s - 1 + n), 0.0) + acc
    sigma = np.zeros((3, 3))
    inv_tau = []
    for kk, k in enumerate(kept):
        s, t = win[k]
        for n in range(s - 1, t):
            it = sout.get((k, n), 0.0)
            inv_tau.append(it)
            if it <= 0:
                continue
            df = -O._occ_fd_deriv(E[n, k] - mu, temp) / it
            vv = V[:, n, kk]
            sigma += (1.0 / N) * df * np.outer(vv, vv)
    return sigma * spin / volume, np.array(inv_tau), dict(kept=kept, E=E, win=win, npairs=npairs)
