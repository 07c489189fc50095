"""EPW model reader (host side of src/model_new.jl:1-568, load_model_from_epw_new).

The text files (crystal.fmt, wigner.fmt, epwdata.fmt) are parsed here as the reference parses them
(GNU and Intel Fortran list-directed layouts, old and new (`-2`) wigner.fmt); the binary
`<prefix>.epmatwp`, which holds gigabytes, is streamed into HBM by the library's `epb_read_epmat`, which
applies the R sort, the Wigner-Seitz divisions and the "el" / "ph" layout on the device. Position,
velocity, polar and symmetry data of the reference's Model are outside the hot path and not read.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check
from .wannier import WannierObject, sort_irvec


def pair_to_complex(line):
    """'(re,im)' -> complex (src/model_new.jl:3-6)."""
    a, b = line.strip()[1:-1].split(",")
    return complex(float(a), float(b))


def parse_wigner(lines, nr, dims1, dims2, skip_ndegen=False):
    """(irvec (nr, 3), ndegen (dims1, dims2, nr) Fortran order, wslen) (src/model_new.jl:8-32)."""
    irvec = np.zeros((nr, 3), dtype=np.int64)
    wslen = np.zeros(nr)
    ndegen = np.zeros((dims1, dims2, nr), dtype=np.int32, order="F")
    for ir in range(nr):
        t = next(lines).split()
        irvec[ir] = [int(x) for x in t[:3]]
        wslen[ir] = float(t[3])
        if not skip_ndegen:
            for i in range(dims1):
                ndegen[i, :, ir] = [int(x) for x in next(lines).split()]
    return irvec, ndegen, wslen


def parse_structure(folder):
    """crystal.fmt (src/model_new.jl:40-160): lattice (bohr, columns a_i), per-atom masses, atom
    positions, nmodes, ws_method, ndegen_pre_divided."""
    with open(os.path.join(folder, "crystal.fmt")) as fh:
        lines = iter(fh.read().splitlines())
    nat = int(next(lines))
    nmodes = int(next(lines))
    float(next(lines).split()[0])  # nelec
    data = next(lines).split()
    if len(data) == 9:
        at = np.array([float(x) for x in data])
        next(lines)  # bg
        gnu = True
    else:
        data += next(lines).split() + next(lines).split()
        at = np.array([float(x) for x in data])
        for _ in range(3):
            next(lines)
        gnu = False
    float(next(lines))  # omega
    alat = float(next(lines))
    if gnu:
        tau = [float(x) for x in next(lines).split()]
        amass = [float(x) for x in next(lines).split()]
        ityp = [int(x) for x in next(lines).split()]
    else:
        tau = sum(([float(x) for x in next(lines).split()] for _ in range(nat)), [])
        amass = sum(([float(x) for x in next(lines).split()] for _ in range(4)), [])
        data = next(lines).split()
        for _ in range((nat - 1) // 6):
            data += next(lines).split()
        ityp = [int(x) for x in data]
    next(lines)  # noncolin
    next(lines)  # do_cutoff_2D_epw
    if gnu:
        next(lines)  # Wannier centers
        float(next(lines))  # L
    else:
        while True:
            d = next(lines).split()
            if len(d) == 1:
                break
            if len(d) != 3:
                raise ValueError("Unexpected line in crystal.fmt")
    ws_method, idiv = -1, 0
    rest = list(lines)
    if rest and rest[0].strip():
        if len(rest) >= 3 and len(rest[2].split()) == 2:
            ws_method, idiv = (int(x) for x in rest[2].split())
            if idiv != 1:
                raise ValueError("idiv must be 1 in crystal.fmt")
    lattice = at.reshape(3, 3, order="F") * alat
    mass_atom = np.array([amass[t - 1] for t in ityp])
    return dict(nat=nat, nmodes=nmodes, lattice=lattice, alat=alat, mass_atom=mass_atom,
                atom_pos=np.array(tau).reshape(3, nat, order="F"), ws_method=ws_method,
                ndegen_pre_divided=(idiv == 1))


def read_wigner(folder, ws_method, ndegen_pre_divided):
    with open(os.path.join(folder, "wigner.fmt")) as fh:
        lines = iter(fh.read().splitlines())
    first = next(lines).split()
    skip_eph_ndegen = False
    if int(first[0]) == -2:  # use_ws_v2
        if not ndegen_pre_divided:
            raise ValueError("wigner.fmt of the new format needs ndegen pre-divided (crystal.fmt idiv = 1)")
        _, wsm, pre = (int(x) for x in first)
        if wsm != ws_method or pre != 1:
            raise ValueError("wigner.fmt and crystal.fmt disagree on the Wigner-Seitz method")
        skip_eph_ndegen = ws_method == 3
        next(lines)  # nw nat
        nr_el, nr_ph, nr_ep, dims, dims2 = (int(x) for x in next(lines).split())
        next(lines)  # coarse grids
    else:
        nr_el, nr_ph, nr_ep, dims, dims2 = (int(x) for x in first)
    el = parse_wigner(lines, nr_el, dims, dims)
    ph = parse_wigner(lines, nr_ph, dims2, dims2)
    ep = parse_wigner(lines, nr_ep, dims, dims2, skip_ndegen=skip_eph_ndegen)
    return dict(nr_el=nr_el, nr_ph=nr_ph, nr_ep=nr_ep, dims=dims, dims2=dims2, el=el, ph=ph, ep=ep,
                skip_eph_ndegen=skip_eph_ndegen)


def _cdiv(z, d):
    """z / d for an integer d with both parts divided, as Julia's Complex / Real."""
    out = np.empty_like(z)
    out.real = z.real / d
    out.imag = z.imag / d
    return out


def _divide(op, ndegen, block=1):
    """op (n, n, nr) /= ndegen per R (1 x 1) or per (i, j) block of size `block` (zero where 0)."""
    out = op.copy()
    if ndegen.shape[0] == 1:
        for ir in range(op.shape[2]):
            d = ndegen[0, 0, ir]
            out[:, :, ir] = 0 if d == 0 else _cdiv(out[:, :, ir], d)
    else:
        n = ndegen.shape[0]
        for ir in range(op.shape[2]):
            for j in range(n):
                for i in range(n):
                    d = ndegen[i, j, ir]
                    s = (slice(block * i, block * i + block), slice(block * j, block * j + block), ir)
                    out[s] = 0 if d == 0 else _cdiv(out[s], d)
    return out


@dataclass
class EpwModel:
    """The fields of the reference `Model` (src/model.jl:24-85) that the hot path reads."""

    nw: int
    nmodes: int
    mass: np.ndarray          # (nmodes,) per Cartesian mode
    lattice: np.ndarray
    el_ham: WannierObject
    ph_dyn: WannierObject
    epmat: object              # device-only two-stage object, or None
    epmat_outer_momentum: str
    ef: float


def load_model_from_epw(folder, outdir, prefix, *, epmat_outer_momentum="el", load_epmat=True,
                        skip_eph_ndegen=False, ctx=None):
    """load_model_from_epw_new (src/model_new.jl:175-484) restricted to H, D, masses and g(Re, Rp)."""
    import torch

    from .synth import DeviceOnlyWannierObject

    if epmat_outer_momentum not in ("el", "ph"):
        raise ValueError("epmat_outer_momentum must be ph or el.")
    st = parse_structure(folder)
    pre = st["ndegen_pre_divided"]
    w = read_wigner(folder, st["ws_method"], pre)
    skip_ep = skip_eph_ndegen or w["skip_eph_ndegen"]
    irvec_el, ndegen_el, _ = w["el"]
    irvec_ph, ndegen_ph, _ = w["ph"]
    irvec_ep, ndegen_ep, _ = w["ep"]
    with open(os.path.join(folder, "epwdata.fmt")) as fh:
        lines = iter(fh.read().splitlines())
    ef = float(next(lines))
    nw, nr_el, nmodes, nr_ph, nr_ep = (int(x) for x in next(lines).split())
    zs = next(lines).split()
    nat = st["nat"]
    if len(zs) == 3:
        for _ in range(3 * nat + 2):
            zs += next(lines).split()
    if len(zs) != 9 * nat + 9:
        raise ValueError("epwdata.fmt: unexpected Born charge / dielectric block")
    ham = np.zeros((nw, nw, nr_el), dtype=np.complex128, order="F")
    for i in range(nw):
        for j in range(nw):
            for ir in range(nr_el):
                ham[i, j, ir] = pair_to_complex(next(lines))
    dyn = np.zeros((nmodes, nmodes, nr_ph), dtype=np.complex128, order="F")
    for i in range(nmodes):
        for j in range(nmodes):
            for ir in range(nr_ph):
                dyn[i, j, ir] = pair_to_complex(next(lines))
    if not pre:
        ham = _divide(ham, ndegen_el)
        dyn = _divide(dyn, ndegen_ph, block=3)
    if np.linalg.norm(dyn) < np.finfo(float).eps:
        raise ValueError("Dynamical matrix is not written in epwdata.fmt. Set lifc = .false. in EPW.")
    ind_el, ind_ph, ind_ep = sort_irvec(irvec_el), sort_irvec(irvec_ph), sort_irvec(irvec_ep)
    ndegen_el, ndegen_ep = ndegen_el[:, :, ind_el], ndegen_ep[:, :, ind_ep]
    el_ham = WannierObject(irvec_el[ind_el], np.asfortranarray(ham[:, :, ind_el].reshape(nw * nw, nr_el, order="F")))
    ph_dyn = WannierObject(irvec_ph[ind_ph], np.asfortranarray(dyn[:, :, ind_ph].reshape(nmodes * nmodes, nr_ph,
                                                                                        order="F")))
    ep = None
    if load_epmat:
        ctx = ctx or _lib.default_context()
        nd = nw * nw * nmodes
        layout = 0 if epmat_outer_momentum == "el" else 1
        out = torch.empty((nr_el, nd * nr_ep) if layout == 0 else (nr_ep, nd * nr_el), dtype=torch.complex128,
                          device="cuda")
        nel = np.asfortranarray(ndegen_el, dtype=np.int32)
        nep = np.asfortranarray(ndegen_ep, dtype=np.int32)
        ie = np.ascontiguousarray(ind_el + 1, dtype=np.int64)
        ip = np.ascontiguousarray(ind_ep + 1, dtype=np.int64)
        fn = os.path.join(folder, outdir, f"{prefix}.epmatwp").encode()
        check(_lib.lib().epb_read_epmat(ctx.h, fn, nw, nmodes, nr_el, nr_ep, ie.ctypes.data, ip.ctypes.data,
                                        nel.ctypes.data, nel.shape[0], nep.ctypes.data, nep.shape[0], nep.shape[1],
                                        1 if skip_ep else 0, 1 if pre else 0, layout, out.data_ptr()))
        if layout == 0:
            ep = DeviceOnlyWannierObject(out, irvec_el[ind_el], irvec_ep[ind_ep])
        else:
            ep = DeviceOnlyWannierObject(out, irvec_ep[ind_ep], irvec_el[ind_el])
    mass = np.repeat(st["mass_atom"], 3)
    return EpwModel(nw, nmodes, mass, st["lattice"], el_ham, ph_dyn, ep,
                    epmat_outer_momentum if load_epmat else "nothing", ef)
