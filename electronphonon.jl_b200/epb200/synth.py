"""Seeded synthetic Wannier models for the five benchmark configurations.

The reference's test models (Pb, cubic BN EPW artifacts) are not available, so every workload
here is generated from a recorded seed with numpy's PCG64. Complex normals are
CN(0,1) = N(0,1/2) + i N(0,1/2). Lattice vectors are boxes `{-n..n}^3` sorted by `reverse(R)`
(`src/wannier/WannierObject.jl:14-17`), lengths are in lattice units (cubic cell, a = 1).

* Hamiltonian H(R) ~ CN(0,1) exp(-|R|/decay) with H(-R) = H(R)^dagger and H(0) Hermitian, the
  construction of the reference's own GPU test model (`test/test_gpu.jl:280-293`).
* Dynamical matrix from a random spring model on the phonon R grid: every bond (a, b, R) carries a
  random positive semi-definite 3x3 spring K exp(-|R|/decay), added as C_aa(0) += K, C_bb(0) += K,
  C_ab(R) -= K, C_ba(-R) -= K. This imposes the acoustic sum rule and C(-R) = C(R)^T (Hermitian
  D(q)) by construction and keeps D(q) positive semi-definite (real frequencies).
* e-ph matrix g(Re, Rp) ~ CN(0,1) exp(-|Re|/2 - |Rp|/1.5) in the reference's `"el"` layout:
  rows (iw, jw, nu, Rp) with iw fastest, columns Re (`src/model_new.jl:551-565`).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .wannier import WannierObject, sort_irvec

# Rydberg atomic units (src/common/units.jl:17-31).
UNIT_EV = 0.03674932248 * 2
UNIT_MEV = UNIT_EV * 1e-3
AMU_RY = 1822.888486209 / 2.0  # atomic mass unit in Rydberg mass units (2 m_e)


def irvec_box(n: int) -> np.ndarray:
    """All R in {-n..n}^3, sorted by reverse(R) (R1 fastest)."""
    r = np.arange(-n, n + 1)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    return np.ascontiguousarray(g[sort_irvec(g)]).astype(np.int64)


def cnormal(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * np.sqrt(0.5)


def hermitian_op_r(rng, nw: int, irvec: np.ndarray, decay: float, scale: float = 1.0) -> np.ndarray:
    """(nw^2, nr) column-major op_r of H(R) ~ CN(0,1) e^{-|R|/decay}, H(-R) = H(R)^dagger."""
    nr = irvec.shape[0]
    index = {tuple(r): i for i, r in enumerate(irvec)}
    op = np.zeros((nw, nw, nr), dtype=np.complex128, order="F")
    for i, r in enumerate(irvec):
        j = index[tuple(-r)]
        if j < i:
            continue
        a = cnormal(rng, (nw, nw)) * (scale * np.exp(-np.linalg.norm(r) / decay))
        if j == i:
            a = (a + a.conj().T) / 2
            op[:, :, i] = a
        else:
            op[:, :, i] = a
            op[:, :, j] = a.conj().T
    return np.asfortranarray(op.reshape(nw * nw, nr, order="F"))


def spring_dynmat_op_r(rng, natom: int, irvec: np.ndarray, decay: float, stiffness: float):
    """(nm^2, nr) real-valued dynamical-matrix op_r (force constants) of a random spring model."""
    nm = 3 * natom
    nr = irvec.shape[0]
    index = {tuple(r): i for i, r in enumerate(irvec)}
    i0 = index[(0, 0, 0)]
    c = np.zeros((nm, nm, nr))
    for ir, r in enumerate(irvec):
        for a in range(natom):
            for b in range(natom):
                # one representative per unordered bond {(a,b,R), (b,a,-R)}
                jr = index[tuple(-r)]
                if (a, b, ir) > (b, a, jr) or (a == b and ir == jr):
                    continue
                bmat = rng.standard_normal((3, 3))
                k = bmat @ bmat.T / 3.0 * stiffness * np.exp(-np.linalg.norm(r) / decay)
                sa, sb = slice(3 * a, 3 * a + 3), slice(3 * b, 3 * b + 3)
                c[sa, sa, i0] += k
                c[sb, sb, i0] += k
                c[sa, sb, ir] -= k
                c[sb, sa, jr] -= k.T
    return np.asfortranarray(c.reshape(nm * nm, nr, order="F").astype(np.complex128))


def epmat_el_op_r(rng, nw, nm, irvec_el, irvec_ep, decay_e=2.0, decay_p=1.5, dtype=np.complex128):
    """(nw^2*nm*nr_ep, nr_el) op_r of g(Re,Rp) in the "el" layout (model_new.jl:561-563)."""
    nr_el, nr_ep = irvec_el.shape[0], irvec_ep.shape[0]
    ndata = nw * nw * nm * nr_ep
    fp = np.exp(-np.linalg.norm(irvec_ep, axis=1) / decay_p)           # (nr_ep,)
    row_scale = np.repeat(fp, nw * nw * nm)                               # rows (iw,jw,nu,Rp)
    op = np.empty((ndata, nr_el), dtype=dtype, order="F")
    for ie in range(nr_el):
        fe = np.exp(-np.linalg.norm(irvec_el[ie]) / decay_e)
        op[:, ie] = cnormal(rng, ndata) * (row_scale * fe)
    return op


@dataclass
class SynthModel:
    """The fields of the reference `Model` (src/model.jl:24-85) that the hot path reads."""

    nw: int
    nmodes: int
    mass: np.ndarray            # (nmodes,) Rydberg mass units, per Cartesian mode
    el_ham: WannierObject       # H(R): (nw^2, nr_el)
    ph_dyn: WannierObject       # D(R): (nm^2, nr_ph)
    epmat: WannierObject | None  # g(Re,Rp), "el" layout, irvec_next = Rp grid
    seed: int


def make_model(nw, natom, n_el, n_ph, seed, *, h_decay=1.5, with_epmat=True,
               fc_decay=1.2, stiffness=0.02):
    rng = np.random.default_rng(seed)
    irvec_el = irvec_box(n_el)
    irvec_ph = irvec_box(n_ph)
    ham = WannierObject(irvec_el, hermitian_op_r(rng, nw, irvec_el, h_decay))
    nm = 3 * natom
    masses_atom = rng.uniform(10.0, 30.0, natom) * AMU_RY
    mass = np.repeat(masses_atom, 3)
    dyn = WannierObject(irvec_ph, spring_dynmat_op_r(rng, natom, irvec_ph, fc_decay, stiffness))
    ep = None
    if with_epmat:
        op = epmat_el_op_r(rng, nw, nm, irvec_el, irvec_ph)
        ep = WannierObject(irvec_el, op, irvec_next=irvec_ph)
    return SynthModel(nw, nm, mass, ham, dyn, ep, seed)


def random_kpoints(n, seed):
    """(3, n) column-major crystal coordinates uniform in [0,1)^3."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.random((3, n)))


def grid_kpoints(ngrid, shift=(0.0, 0.0, 0.0)):
    """Regular grid, k fastest (`src/common/kpoints.jl:135-153`); returns (3, nk)."""
    n1, n2, n3 = ngrid
    ik = np.arange(n1 * n2 * n3)
    k = ik % n3
    j = (ik // n3) % n2
    i = ik // (n2 * n3)
    x = np.stack([i / n1, j / n2, k / n3]) + np.asarray(shift, dtype=float)[:, None]
    return np.asfortranarray(x)


# Configuration table (sizes as named by the benchmark definitions).
CONFIGS = {
    1: dict(nw=8, natom=0, n_el=3, n_ph=0, nk=4096, nq=0),
    2: dict(nw=16, natom=4, n_el=4, n_ph=2, nk=2048, nq=8192),
    4: dict(nw=32, natom=4, n_el=5, n_ph=2, nk=96 ** 3, nq=8192),
}


def config1(seed=1):
    rng = np.random.default_rng(seed)
    irvec = irvec_box(3)
    ham = WannierObject(irvec, hermitian_op_r(rng, 8, irvec, 1.5))
    return ham, random_kpoints(4096, seed + 1000)


def config2_model(seed=2, *, with_epmat=True, n_el=4, n_ph=2, nw=16, natom=4):
    return make_model(nw, natom, n_el, n_ph, seed, with_epmat=with_epmat)


def config3_matrices(count, seed=3, sizes=None, degenerate_frac=0.05, spacing=1e-10):
    """Uneven batch of Hermitian matrices: n ~ U{4,8,...,96}; a fraction with planted 2-4-fold
    clusters spaced `spacing` (Q diag Q^dagger construction). Returns (list of n, list of arrays)."""
    rng = np.random.default_rng(seed)
    if sizes is None:
        sizes = np.arange(4, 97, 4)
    ns = rng.choice(sizes, count)
    mats = []
    for n in ns:
        if rng.random() < degenerate_frac:
            ev = np.sort(rng.standard_normal(n) * np.sqrt(n))
            c = int(rng.integers(2, 5))
            c = min(c, n)
            start = int(rng.integers(0, n - c + 1))
            ev[start:start + c] = ev[start] + spacing * np.arange(c)
            q, _ = np.linalg.qr(cnormal(rng, (n, n)))
            a = (q * ev) @ q.conj().T
            a = (a + a.conj().T) / 2
        else:
            a = cnormal(rng, (n, n))
            a = (a + a.conj().T) / 2
        mats.append(np.asfortranarray(a))
    return ns.astype(np.int64), mats


def epmat_el_device(seed, nw, nm, irvec_el, irvec_ep, decay_e=2.0, decay_p=1.5, device="cuda"):
    """g(Re,Rp) of the "el" layout generated on the GPU with torch's seeded Philox generator
    (same distribution as `epmat_el_op_r`; used for the 4.5 GB full-size workload, where host
    generation would dominate start-up). Returns a complex128 tensor of shape (nr_el, ndata), i.e.
    the column-major (ndata, nr_el) operator."""
    import torch

    nr_el, nr_ep = irvec_el.shape[0], irvec_ep.shape[0]
    ndata = nw * nw * nm * nr_ep
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    out = torch.randn((nr_el, ndata), dtype=torch.complex128, device=device, generator=g)  # CN(0,1)
    fe = torch.as_tensor(np.exp(-np.linalg.norm(irvec_el, axis=1) / decay_e), device=device)
    fp = torch.as_tensor(np.repeat(np.exp(-np.linalg.norm(irvec_ep, axis=1) / decay_p), nw * nw * nm), device=device)
    out *= fe[:, None]
    out *= fp[None, :]
    return out


class DeviceOnlyWannierObject:
    """A two-stage operator whose op_r exists only on the device (full-size generated workloads)."""

    def __init__(self, op_dev, irvec, irvec_next):
        self.op_r = op_dev
        self.irvec = np.ascontiguousarray(irvec, dtype=np.int64)
        self.irvec_next = np.ascontiguousarray(irvec_next, dtype=np.int64)
        self.nr = self.irvec.shape[0]
        self.ndata = op_dev.shape[1]


def device_epmat_object(op_dev, irvec_el, irvec_ep):
    return DeviceOnlyWannierObject(op_dev, irvec_el, irvec_ep)
