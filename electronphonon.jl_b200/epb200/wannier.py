"""Host-side mirror of the reference's real-space operator container.

`WannierObject` follows ElectronPhonon.jl `src/wannier/WannierObject.jl:22-70`: an operator
`op_r` of shape `(ndata, nr)` (column-major, complex128) over the lattice vectors `irvec`
(`nr x 3`, integer), sorted by the reversed vector (`WannierObject.jl:14-17`). `ndata` may be
smaller than `op_r.shape[0]` (partial transform). `irvec_next` holds the second-stage lattice
vectors of a two-stage object (the e-ph matrix `g(Re, Rp)`, `model_new.jl:551-565`).

`to_device` mirrors `ext/ElectronPhononCUDAExt.jl:51-53`: the operator moves to the GPU once,
`irvec` stays on the host (a device copy is kept as int64 for the kernels).
"""
from __future__ import annotations

import numpy as np


def sort_irvec(irvec):
    """Permutation sorting lattice vectors by `reverse(R)` (`WannierObject.jl:46-52`)."""
    irvec = np.asarray(irvec)
    return np.lexsort((irvec[:, 0], irvec[:, 1], irvec[:, 2]))


def irvec_is_sorted(irvec) -> bool:
    """`issorted(irvec, by=x->reverse(x))` (`WannierObject.jl:14`)."""
    irvec = np.asarray(irvec)
    keys = irvec[:, ::-1]
    for a, b in zip(keys[:-1], keys[1:]):
        if tuple(a) > tuple(b):
            return False
    return True


class WannierObject:
    """Real-space operator `op_r[ndata, nr]` over `irvec` (see module docstring).

    `op_r` is either a numpy array (host) or a torch tensor (device, complex128, column-major
    i.e. stored as the transpose-contiguous layout expected by the C ABI).
    """

    def __init__(self, irvec, op_r, *, irvec_next=None, sort=False, ndata=None):
        irvec = np.ascontiguousarray(np.asarray(irvec, dtype=np.int64).reshape(-1, 3))
        if sort:
            perm = sort_irvec(irvec)
            irvec = irvec[perm]
            op_r = op_r[:, perm]
        if op_r.shape[1] != irvec.shape[0]:
            raise ValueError(f"size(op_r, 2)={op_r.shape[1]} must equal length(irvec)={irvec.shape[0]}")
        if not irvec_is_sorted(irvec):
            raise ValueError("irvec is not sorted. irvec must be sorted by reverse(r)")
        self.irvec = irvec
        self.nr = irvec.shape[0]
        self.op_r = op_r
        self.ndata = op_r.shape[0] if ndata is None else int(ndata)
        if not (1 <= self.ndata <= op_r.shape[0]):
            raise ValueError(f"ndata={self.ndata} must be in 1:{op_r.shape[0]}")
        self.irvec_next = None if irvec_next is None else np.ascontiguousarray(
            np.asarray(irvec_next, dtype=np.int64).reshape(-1, 3))
        self._id = 0
        self._irvec_dev = None

    @property
    def on_device(self) -> bool:
        return not isinstance(self.op_r, np.ndarray)

    def __repr__(self):
        return f"WannierObject(nr={self.nr}, ndata={self.ndata}, device={self.on_device})"


def to_device(obj: WannierObject, device="cuda"):
    """Copy of a host `obj` with `op_r` on the GPU (`ext/ElectronPhononCUDAExt.jl:51-53`).

    The device operator is stored column-major: a torch tensor of shape `(nr, ndata_full)`
    whose row `r` is column `r` of `op_r`, i.e. exactly the bytes of the Julia `CuMatrix`.
    """
    import torch

    if obj.on_device:
        raise TypeError("to_device is defined for host objects only")
    host = np.asfortranarray(obj.op_r.astype(np.complex128, copy=False))
    dev = torch.from_numpy(np.ascontiguousarray(host.T)).to(device)
    out = WannierObject.__new__(WannierObject)
    out.irvec = obj.irvec
    out.nr = obj.nr
    out.op_r = dev
    out.ndata = obj.ndata
    out.irvec_next = obj.irvec_next
    out._id = 0
    # (nr, 3) C-contiguous int64 == Julia's Vector{Vec3{Int}} bytes (3 x nr column-major).
    out._irvec_dev = torch.from_numpy(np.ascontiguousarray(obj.irvec)).to(device)
    return out
