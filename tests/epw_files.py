"""Writer of EPW-format model folders (crystal.fmt, wigner.fmt, epwdata.fmt, <prefix>.epmatwp) from a
synthetic model, in the layouts the reference parses (src/model_new.jl): used by tests/test_epw.py to
round-trip the reader. R vectors are written in a shuffled (unsorted) order with Wigner-Seitz
degeneracies, and the stored matrix elements are multiplied by them, as EPW writes undivided data."""
from __future__ import annotations

import os

import numpy as np


def _pair(z):
    return f"({float(z.real)!r},{float(z.imag)!r})"


def write_epw_folder(folder, model, natom, *, seed=0, intel=False, new_wigner=False, ws_method=2,
                     ndegen_per_orbital=True, zero_ndegen=False, prefix="test", outdir="out"):
    rng = np.random.default_rng(seed)
    nw, nm = model.nw, model.nmodes
    ham, dyn, ep = model.el_ham, model.ph_dyn, model.epmat
    irvec_el, irvec_ph, irvec_ep = ham.irvec, dyn.irvec, ep.irvec_next
    nr_el, nr_ph, nr_ep = len(irvec_el), len(irvec_ph), len(irvec_ep)
    # file order: a shuffle of the sorted lists
    p_el, p_ph, p_ep = rng.permutation(nr_el), rng.permutation(nr_ph), rng.permutation(nr_ep)
    pre = new_wigner
    dims = nw if ndegen_per_orbital else 1
    dims2 = natom if ndegen_per_orbital else 1
    nd_el = rng.integers(1, 4, (dims, dims, nr_el)).astype(np.int32)
    nd_ph = rng.integers(1, 4, (dims2, dims2, nr_ph)).astype(np.int32)
    nd_ep = rng.integers(1, 4, (dims, dims2, nr_ep)).astype(np.int32)
    if zero_ndegen:
        nd_el[..., 1] = 0
        nd_ep[..., 2] = 0
    skip_ep = new_wigner and ws_method == 3
    if pre:
        f_el = np.ones((nw, nw, nr_el))
        f_ph = np.ones((nm, nm, nr_ph))
        f_ep_el = np.ones((nw, nw, nr_el))
        f_ep_ep = np.ones((nw, nm, nr_ep))
    else:
        f_el = np.broadcast_to(nd_el if dims > 1 else nd_el[0, 0][None, None, :], (nw, nw, nr_el)).astype(float)
        f_ph = (np.repeat(np.repeat(nd_ph, 3, 0), 3, 1) if dims2 > 1 else np.broadcast_to(nd_ph[0, 0][None, None, :],
                                                                                          (nm, nm, nr_ph))).astype(float)
        f_ep_el = f_el
        f_ep_ep = (np.repeat(nd_ep, 3, 1) if dims > 1 else np.broadcast_to(nd_ep[0, 0][None, None, :],
                                                                           (nw, nm, nr_ep))).astype(float)
    os.makedirs(os.path.join(folder, outdir), exist_ok=True)
    # crystal.fmt
    lat = np.eye(3)
    alat = 1.0
    mass_atom = model.mass[::3]
    with open(os.path.join(folder, "crystal.fmt"), "w") as fh:
        w = lambda vals: fh.write(" ".join(repr(float(v)) for v in vals) + "\n")
        fh.write(f"{natom}\n{nm}\n{2.0 * nw!r}\n")
        at = lat.reshape(-1, order="F")
        bg = np.linalg.inv(lat).T.reshape(-1, order="F")
        if intel:
            for i in range(3):
                w(at[3 * i:3 * i + 3])
            for i in range(3):
                w(bg[3 * i:3 * i + 3])
        else:
            w(at)
            w(bg)
        fh.write("1.0\n")
        fh.write(f"{alat!r}\n")
        tau = rng.random((3, natom))
        amass = np.zeros(10)
        amass[:natom] = mass_atom
        ityp = np.arange(1, natom + 1)
        if intel:
            for a in range(natom):
                w(tau[:, a])
            w(amass[0:3]), w(amass[3:6]), w(amass[6:9]), w(amass[9:10])
            for c in range(0, natom, 6):
                fh.write(" ".join(str(int(t)) for t in ityp[c:c + 6]) + "\n")
        else:
            w(tau.reshape(-1, order="F"))
            w(amass)
            fh.write(" ".join(str(int(t)) for t in ityp) + "\n")
        fh.write("F\nF\n")
        centers = rng.random((3, nw))
        if intel:
            for i in range(nw):
                w(centers[:, i])
        else:
            w(centers.reshape(-1, order="F"))
        fh.write("0.0\n")
        if new_wigner:
            fh.write("0.01\n0\n")
            fh.write(f"{ws_method} 1\n")
    # wigner.fmt
    with open(os.path.join(folder, "wigner.fmt"), "w") as fh:
        if new_wigner:
            fh.write(f"-2 {ws_method} 1\n{nw} {natom}\n{nr_el} {nr_ph} {nr_ep} {dims} {dims2}\n4 4 4 4 4 4\n")
        else:
            fh.write(f"{nr_el} {nr_ph} {nr_ep} {dims} {dims2}\n")
        for irv, perm, nd, d1, skip in ((irvec_el, p_el, nd_el, dims, False), (irvec_ph, p_ph, nd_ph, dims2, False),
                                        (irvec_ep, p_ep, nd_ep, dims, skip_ep)):
            for i in perm:
                r = irv[i]
                fh.write(f"{r[0]} {r[1]} {r[2]} {float(np.linalg.norm(r))!r}\n")
                if not skip:
                    for a in range(d1):
                        fh.write(" ".join(str(int(x)) for x in nd[a, :, i]) + "\n")
    # epwdata.fmt
    H = ham.op_r.reshape(nw, nw, nr_el, order="F")
    D = dyn.op_r.reshape(nm, nm, nr_ph, order="F")
    with open(os.path.join(folder, "epwdata.fmt"), "w") as fh:
        fh.write("0.5\n")
        fh.write(f"{nw} {nr_el} {nm} {nr_ph} {nr_ep}\n")
        fh.write(" ".join(["0.0"] * (9 * natom + 9)) + "\n")
        for i in range(nw):
            for j in range(nw):
                for k in p_el:
                    fh.write(_pair(H[i, j, k] * f_el[i, j, k]) + "\n")
        for i in range(nm):
            for j in range(nm):
                for k in p_ph:
                    fh.write(_pair(D[i, j, k] * f_ph[i, j, k]) + "\n")
    # <prefix>.epmatwp: (iw, jw, iRe, imode, iRp) in file R order
    G = np.asarray(ep.op_r).reshape(nw, nw, nm, nr_ep, nr_el, order="F")  # "el" layout, sorted
    raw = np.empty((nw, nw, nr_el, nm, nr_ep), dtype=np.complex128, order="F")
    for a, ie in enumerate(p_el):
        for b, ip in enumerate(p_ep):
            blk = G[:, :, :, ip, ie]  # (nw, nw, nm)
            fac = f_ep_el[:, :, ie][:, :, None] * (1.0 if skip_ep else f_ep_ep[:, :, ip][:, None, :])
            raw[:, :, a, :, b] = blk * fac
    raw.reshape(-1, order="F").tofile(os.path.join(folder, outdir, f"{prefix}.epmatwp"))
    return dict(p_el=p_el, p_ph=p_ph, p_ep=p_ep, nd_el=nd_el, nd_ph=nd_ph, nd_ep=nd_ep, dims=dims, dims2=dims2,
                skip_ep=skip_ep, pre=pre)
