"""Band energies, energy windows and the learned pre-filter (host mirror over libepb200).

`BandModel` binds an electron Hamiltonian H(R) for eigenvalue-only queries (the role of
`get_el_eigen_valueonly_batched`, `src/wannier_to_bloch_batched.jl:75-88`) and for the energy-window
tests of `src/filter.jl:19,40-72` and of the (k, q) pair loop
(`src/calculator/run_eph_over_k_and_q.jl:303-307`). `Surrogate` is the MLP pre-filter: trained
on band energies of the plain path by the library's own kernels, calibrated on held-out points,
then used by `pair_window` to cull pairs whose every band is predicted outside the window by more
than the calibrated margin. `learned_pair_filter` runs the whole workflow.

All compute runs in libepb200.so; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import PREC_FP64, PREC_MIXED, MlpTrainOpts, WindowStats, check, ptr  # noqa: F401
from .batched import _xk_dev, jl_empty
from .wannier import WannierObject, to_device

DEFAULT_GUARD = 1e-3  # Ry: the mixed path re-evaluates in FP64 any point with a band this close to an edge


def _torch():
    import torch

    return torch


def _ctx():
    return _lib.default_context()


def feature_vectors(nf: int) -> np.ndarray:
    """The nf shortest nonzero integer vectors of one half-space (f and -f give the same features up
    to sign), ordered by |f|^2 then lexicographically; int32 (3, nf) column-major."""
    r = 1
    while (2 * r + 1) ** 3 // 2 < nf:
        r += 1
    g = np.arange(-r, r + 1)
    f = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = (f[:, 0] > 0) | ((f[:, 0] == 0) & (f[:, 1] > 0)) | ((f[:, 0] == 0) & (f[:, 1] == 0) & (f[:, 2] > 0))
    f = f[pos]
    order = np.lexsort((f[:, 2], f[:, 1], f[:, 0], (f * f).sum(1)))
    return np.asfortranarray(f[order[:nf]].T.astype(np.int32))


# ---------------------------------------------------------------------------------------------
class BandModel:
    """epb_bands: H(R) on the device plus its tensor-core operand planes."""

    def __init__(self, ham: WannierObject):
        self.ham_host_op = None if ham.on_device else ham.op_r
        if not ham.on_device:
            ham = to_device(ham)
        self.ham = ham
        self.nw = int(round(np.sqrt(ham.ndata)))
        assert self.nw * self.nw == ham.ndata
        self.ctx = _ctx()
        h = C.c_void_p()
        irv = np.ascontiguousarray(ham.irvec, dtype=np.int64)
        check(_lib.lib().epb_bands_create(self.ctx.h, ptr(ham.op_r), self.nw, irv.ctypes.data, ham.nr, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().epb_bands_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def eigvals(self, xks, prec=PREC_FP64):
        """Ascending band energies, device (nw, nk) in Julia layout (torch shape (nk, nw))."""
        torch = _torch()
        x = _xk_dev(xks)
        nk = x.numel() // 3
        E = jl_empty((self.nw, nk), torch.float64)
        check(_lib.lib().epb_bands_eigvals(self.ctx.h, self.h, ptr(x), nk, ptr(E), prec))
        return E

    def band_energy(self, xks, band, prec=PREC_FP64):
        """Energy of band `band` (1-based) at every point, device (nk,)."""
        torch = _torch()
        x = _xk_dev(xks)
        nk = x.numel() // 3
        E = torch.empty(nk, dtype=torch.float64, device=x.device)
        check(_lib.lib().epb_bands_band_energy(self.ctx.h, self.h, ptr(x), nk, int(band), ptr(E), prec))
        return E

    def window(self, xks, wmin, wmax, prec=PREC_FP64, guard=DEFAULT_GUARD):
        """(band_min, band_max, keep_idx, stats) of every point (1-based ranges, 0-based keep list)."""
        torch = _torch()
        x = _xk_dev(xks)
        nk = x.numel() // 3
        bmin = torch.empty(nk, dtype=torch.int32, device=x.device)
        bmax = torch.empty(nk, dtype=torch.int32, device=x.device)
        keep = torch.empty(max(nk, 1), dtype=torch.int32, device=x.device)
        nkeep = C.c_int64()
        st = WindowStats()
        check(_lib.lib().epb_bands_window(self.ctx.h, self.h, ptr(x), nk, float(wmin), float(wmax), prec, float(guard),
                                          ptr(bmin), ptr(bmax), ptr(keep), C.byref(nkeep), C.byref(st)))
        return bmin, bmax, keep[:nkeep.value], st.as_dict()


# ---------------------------------------------------------------------------------------------
class Surrogate:
    """epb_mlp: Fourier-feature MLP predicting the nout band energies of a point."""

    def __init__(self, nf=128, hidden=256, nhidden=3, nout=32, seed=0):
        self.ctx = _ctx()
        self.fvec = feature_vectors(nf)
        h = C.c_void_p()
        check(_lib.lib().epb_mlp_create(self.ctx.h, self.fvec.ctypes.data, nf, hidden, nhidden, nout, int(seed),
                                        C.byref(h)))
        self.h = h
        npar, nin, no = C.c_int64(), C.c_int64(), C.c_int64()
        check(_lib.lib().epb_mlp_info(self.h, C.byref(npar), C.byref(nin), C.byref(no)))
        self.nparam, self.nin, self.nout = npar.value, nin.value, no.value
        self.nf, self.hidden, self.nhidden = nf, hidden, nhidden
        self.margin = None
        self.history = []

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().epb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters and normalisation
    def get_params(self):
        torch = _torch()
        p = torch.empty(self.nparam, dtype=torch.float32, device="cuda")
        check(_lib.lib().epb_mlp_get_params(self.ctx.h, self.h, ptr(p)))
        return p

    def set_params(self, p):
        torch = _torch()
        p = torch.as_tensor(p, dtype=torch.float32, device="cuda").contiguous()
        assert p.numel() == self.nparam
        check(_lib.lib().epb_mlp_set_params(self.ctx.h, self.h, ptr(p)))
        self.ctx.synchronize()

    def set_scaling(self, mu, sc):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        sc = np.ascontiguousarray(sc, dtype=np.float64)
        check(_lib.lib().epb_mlp_set_scaling(self.ctx.h, self.h, mu.ctypes.data, sc.ctypes.data))

    def get_scaling(self):
        mu = np.zeros(self.nout)
        sc = np.zeros(self.nout)
        check(_lib.lib().epb_mlp_get_scaling(self.ctx.h, self.h, mu.ctypes.data, sc.ctypes.data))
        return mu, sc

    # kernels
    def features(self, xks):
        torch = _torch()
        x = _xk_dev(xks)
        n = x.numel() // 3
        F = torch.empty((n, self.nin), dtype=torch.float32, device=x.device)
        check(_lib.lib().epb_mlp_features(self.ctx.h, self.h, ptr(x), n, ptr(F)))
        return F

    def loss_grad(self, xks, E):
        """(loss, gradient) of the mean-squared error on the points xks with energies E (nout, n)."""
        torch = _torch()
        x = _xk_dev(xks)
        n = x.numel() // 3
        Ed = E if isinstance(E, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(E).T)).cuda()
        g = torch.empty(self.nparam, dtype=torch.float32, device="cuda")
        loss = C.c_double()
        check(_lib.lib().epb_mlp_loss_grad(self.ctx.h, self.h, ptr(x), ptr(Ed), n, ptr(g), C.byref(loss)))
        return loss.value, g

    def train(self, xks, E, epochs=200, batch=2048, lr=2e-3, lr_final=2e-5, seed=1, use_graph=True):
        """Adam on the points xks with band energies E (device (nout, n) Julia layout or host)."""
        torch = _torch()
        x = _xk_dev(xks)
        n = x.numel() // 3
        Ed = E if isinstance(E, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(E).T)).cuda()
        opts = MlpTrainOpts(epochs=int(epochs), batch=int(batch), lr=float(lr), lr_final=float(lr_final),
                            seed=int(seed), use_graph=1 if use_graph else 0, reserved=0)
        loss = np.zeros(int(epochs))
        check(_lib.lib().epb_mlp_train(self.ctx.h, self.h, ptr(x), ptr(Ed), n, C.byref(opts), loss.ctypes.data))
        self.history = loss
        return loss

    def set_inference(self, mode):
        """1: BF16 tensor cores (default), 0: FP32 kernels. Clears the calibration."""
        check(_lib.lib().epb_mlp_set_inference(self.h, int(mode)))
        self.margin = None

    def inference_path(self):
        v = C.c_int()
        check(_lib.lib().epb_mlp_inference_path(self.h, C.byref(v)))
        return v.value

    def predict(self, xks):
        torch = _torch()
        x = _xk_dev(xks)
        n = x.numel() // 3
        E = jl_empty((self.nout, n), torch.float64)
        check(_lib.lib().epb_mlp_predict(self.ctx.h, self.h, ptr(x), n, ptr(E)))
        return E

    def calibrate(self, xks, E, safety=1.5):
        """Per-band culling margins = safety x max held-out |prediction - E|. The maximum over a few
        10^4 held-out points underestimates the error tail over 10^7-10^8 screened points; the default
        safety of 1.5 covers it on the tested models, and the pair window's audit checks it."""
        torch = _torch()
        x = _xk_dev(xks)
        n = x.numel() // 3
        Ed = E if isinstance(E, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(E).T)).cuda()
        m = np.zeros(self.nout)
        check(_lib.lib().epb_mlp_calibrate(self.ctx.h, self.h, ptr(x), ptr(Ed), n, float(safety), m.ctypes.data))
        self.margin = m
        return m


# ---------------------------------------------------------------------------------------------
def pair_window(bands: BandModel, xks, xqs, wmin, wmax, mlp: Surrogate | None = None, prec=PREC_FP64,
                guard=DEFAULT_GUARD, capacity=None):
    """Kept (k, q) pairs: (pairs p = ik nq + iq ascending, band_min, band_max, stats)."""
    torch = _torch()
    xk = _xk_dev(xks)
    xq = _xk_dev(xqs)
    nk, nq = xk.numel() // 3, xq.numel() // 3
    if capacity is None:
        capacity = nk * nq
    pairs = torch.empty(max(capacity, 1), dtype=torch.int64, device="cuda")
    bmin = torch.empty(max(capacity, 1), dtype=torch.int32, device="cuda")
    bmax = torch.empty(max(capacity, 1), dtype=torch.int32, device="cuda")
    n = C.c_int64()
    st = WindowStats()
    check(_lib.lib().epb_pair_window(bands.ctx.h, bands.h, ptr(xk), nk, ptr(xq), nq, float(wmin), float(wmax),
                                     mlp.h if mlp is not None else None, prec, float(guard), ptr(pairs), ptr(bmin),
                                     ptr(bmax), int(capacity), C.byref(n), C.byref(st)))
    k = n.value
    return pairs[:k], bmin[:k], bmax[:k], st.as_dict()


@dataclass
class LearnedFilterResult:
    e_fermi: float
    wmin: float
    wmax: float
    k_keep: object              # device int32, kept grid k (0-based)
    pairs: object               # device int64, kept pairs p = ik_kept * nq + iq
    band_min: object
    band_max: object
    stats: dict
    margin: np.ndarray
    train_loss: np.ndarray
    timings: dict = field(default_factory=dict)


def learned_pair_filter(bands: BandModel, xk_grid, xqs, half_window, fermi_band, n_train=1 << 15, n_holdout=1 << 16,
                        prec=PREC_MIXED, guard=DEFAULT_GUARD, surrogate=None, train_kw=None, seed=11,
                        use_surrogate=True, capacity=None):
    """The learned-filter workflow: plain window on the k grid (E_F = median of band `fermi_band`
    (1-based) over the grid, window E_F -/+ half_window), surrogate trained on band energies of
    n_train random points and calibrated on n_holdout others, then the (kept k, q) pair window
    with the surrogate pre-filter (or without it when use_surrogate is False)."""
    import time

    torch = _torch()
    t = {}
    t0 = time.perf_counter()
    e_band = bands.band_energy(xk_grid, fermi_band, prec=PREC_FP64)
    ef = float(torch.median(e_band).item())
    wmin, wmax = ef - half_window, ef + half_window
    _, _, k_keep, _ = bands.window(xk_grid, wmin, wmax, prec=prec, guard=guard)
    xk_all = _xk_dev(xk_grid)
    xk_kept = xk_all.index_select(0, k_keep.long()).contiguous()
    torch.cuda.synchronize()
    t["k_grid"] = time.perf_counter() - t0
    margin = np.zeros(bands.nw)
    loss = np.zeros(0)
    mlp = None
    if use_surrogate:
        t0 = time.perf_counter()
        rng = np.random.default_rng(seed)
        xt = np.asfortranarray(rng.random((3, n_train)))
        xh = np.asfortranarray(rng.random((3, n_holdout)))
        Et = bands.eigvals(xt, prec=PREC_FP64)
        Eh = bands.eigvals(xh, prec=PREC_FP64)
        mlp = surrogate or Surrogate(nout=bands.nw, seed=seed)
        loss = mlp.train(xt, Et, **(train_kw or {}))
        margin = mlp.calibrate(xh, Eh)
        torch.cuda.synchronize()
        t["surrogate"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    pairs, bmin, bmax, st = pair_window(bands, xk_kept, xqs, wmin, wmax, mlp=mlp, prec=prec, guard=guard,
                                        capacity=capacity)
    torch.cuda.synchronize()
    t["pairs"] = time.perf_counter() - t0
    return LearnedFilterResult(ef, wmin, wmax, k_keep, pairs, bmin, bmax, st, margin, loss, t)
