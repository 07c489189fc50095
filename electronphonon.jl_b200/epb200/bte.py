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
          volume=1.0, spin=2.0, prec=PREC_FP64, k_batch=0, want_inv_tau=False, inv_tau_cap=None, pair_chunk=0,
          shard=None):
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
    if shard is not None:  # (rank, count): this rank's contiguous share of the kept k; sigma is partial
        p.shard_rank, p.shard_count = int(shard[0]), int(shard[1])
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


def reduce_shards(sigma, stats):
    """Whole-run sigma and counts from this rank's shard result: sigma and the pair / state counts are
    summed over the ranks of the initialised torch.distributed group (one small all-reduce; the kept-k
    count and the window width are the same on every rank). Without a group, returns the inputs."""
    from .shard import _dist

    d = _dist()
    if d is None:
        return sigma, dict(stats)
    import torch

    t = torch.tensor(list(np.asarray(sigma, dtype=np.float64).reshape(-1, order="F")) +
                     [float(stats["pairs"]), float(stats["states"])], dtype=torch.float64)
    if d.get_backend() == "nccl":
        t = t.cuda()
    d.all_reduce(t, op=d.ReduceOp.SUM)
    v = t.cpu().numpy()
    out = dict(stats)
    out["pairs"], out["states"] = int(round(v[9])), int(round(v[10]))
    return v[:9].reshape(3, 3, order="F"), out

