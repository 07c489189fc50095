"""SERTA Boltzmann consumer over commensurate k = q grids (host mirror of epb_bte_serta).

`serta` plays the role of the reference's batched k / k+q loop run with a Boltzmann calculator
followed by the SERTA part of `solve_electron_bte` (src/calculator/run_eph_over_k_and_kq.jl:792-892,
src/boltzmann/boltzmann_calculator.jl:336-362, src/boltzmann/electron_lbte.jl:153-185).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PREC_FP64, BteParams, check, ptr

# src/common/constants.jl:5 (0.01 meV in Ry)
OMEGA_ACOUSTIC = 0.01 * 0.03674932248 * 2 * 1e-3


def serta(dm, ngrid, wmin, wmax, mu, temperature, smearing, method=5, omega_cutoff=OMEGA_ACOUSTIC, lattice=None,
          volume=1.0, spin=2.0, prec=PREC_FP64, k_batch=0, want_inv_tau=False, inv_tau_cap=None, pair_chunk=0):
    """(sigma (3, 3), stats, inv_tau or None) for the model `dm` (pipeline.DeviceModel)."""
    import torch

    p = BteParams()
    p.ngrid = int(ngrid)
    p.wmin, p.wmax, p.mu, p.temperature, p.smearing = float(wmin), float(wmax), float(mu), float(temperature), float(smearing)
    p.omega_cutoff, p.spin_degeneracy, p.volume = float(omega_cutoff), float(spin), float(volume)
    L = np.eye(3) if lattice is None else np.asarray(lattice, dtype=np.float64)
    for i, v in enumerate(np.asarray(L, dtype=np.float64).reshape(-1, order="F")):
        p.lattice[i] = v
    p.method, p.prec, p.k_batch = int(method), int(prec), int(k_batch)
    p.pair_chunk = int(pair_chunk)
    sig = np.zeros(9)
    stats = (C.c_int64 * 4)()
    cap = 0
    it = None
    if want_inv_tau:
        cap = int(inv_tau_cap if inv_tau_cap is not None else ngrid ** 3 * dm.nw)
        it = torch.zeros(max(cap, 1), dtype=torch.float64, device="cuda")
    check(_lib.lib().epb_bte_serta(dm.ctx.h, dm.h, C.byref(p), sig.ctypes.data, ptr(it), cap, stats))
    st = dict(kept_k=stats[0], states=stats[1], pairs=stats[2], width=stats[3])
    return sig.reshape(3, 3, order="F"), st, (it[: st["states"]].cpu().numpy() if want_inv_tau else None)
