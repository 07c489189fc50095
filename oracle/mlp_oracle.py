"""CPU FP64 oracle of the learned window pre-filter (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only `tests/`, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of `bench.py` may import it.

What it restates:
  * the surrogate network of the library (no counterpart in the reference): Fourier features of k,
    SiLU hidden layers, linear output, mean-squared error, its gradient by backpropagation, and one
    Adam step, all in FP64, on the library's flat parameter layout (per layer W (in x out,
    row-major) then b, each block padded to a multiple of 4);
  * the plain energy-window test that the surrogate must never contradict: band energies by LAPACK
    ZHEEV of H(x) = sum_R H(R) e^{2 pi i R.x} (`src/wannier_to_bloch_batched.jl:30-40,75-88`) and the
    in-window range searchsortedfirst(e, wmin) : searchsortedlast(e, wmax) (`src/filter.jl:19`);
    (k, q) pairs kept iff the range at x_k + x_q is non-empty
    (`src/calculator/run_eph_over_k_and_q.jl:303-307`).

Pinning: the window test is the oracle's `inside_window` / `eigvals_batched`, pinned to the
reference's tests in `tests/test_oracle.py`; the network has no reference counterpart and is
pinned by finite-difference gradient checks in `tests/test_mlp.py`.
"""
from __future__ import annotations

import numpy as np

from . import epb_oracle as O


def layer_shapes(nin, hidden, nhidden, nout):
    """[(fan_in, fan_out, w_off, b_off)] and nparam, the library's flat layout."""
    out, off = [], 0
    for l in range(nhidden + 1):
        fi = nin if l == 0 else hidden
        fo = nout if l == nhidden else hidden
        w = off
        off += fi * fo
        b = off
        off += fo
        off = (off + 3) & ~3
        out.append((fi, fo, w, b))
    return out, off


def unpack(params, shapes):
    Ws, bs = [], []
    for fi, fo, w, b in shapes:
        Ws.append(np.asarray(params[w:w + fi * fo], dtype=np.float64).reshape(fi, fo))
        bs.append(np.asarray(params[b:b + fo], dtype=np.float64))
    return Ws, bs


def features(fvec, x):
    """Rows [cos 2 pi f.x, sin 2 pi f.x] per vector f (n x 2 nf); x is (3, n)."""
    t = np.asarray(fvec, dtype=np.float64).reshape(-1, 3) @ np.asarray(x, dtype=np.float64)  # (nf, n)
    t = t - np.rint(t)
    c, s = np.cos(2 * np.pi * t), np.sin(2 * np.pi * t)
    return np.stack([c.T, s.T], axis=-1).reshape(t.shape[1], -1)


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(params, shapes, X):
    """Normalised outputs (n x nout) and the per-layer (input, pre-activation) cache."""
    Ws, bs = unpack(params, shapes)
    cache = []
    h = X
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = h @ W + b
        cache.append((h, z))
        h = z * _sig(z) if l < len(Ws) - 1 else z
    return h, cache


def loss_grad(params, shapes, X, Y):
    """L = sum (out - Y)^2 / (n nout) and dL/dparams (flat, the library's layout)."""
    out, cache = forward(params, shapes, X)
    n, nout = Y.shape
    d = out - Y
    loss = float(np.sum(d * d) / (n * nout))
    g = np.zeros(len(params))
    dz = 2.0 * d / (n * nout)
    Ws, _ = unpack(params, shapes)
    for l in range(len(shapes) - 1, -1, -1):
        fi, fo, w, b = shapes[l]
        h, _ = cache[l]
        g[w:w + fi * fo] = (h.T @ dz).reshape(-1)
        g[b:b + fo] = dz.sum(axis=0)
        if l == 0:
            break
        dh = dz @ Ws[l].T
        zp = cache[l - 1][1]
        s = _sig(zp)
        dz = dh * (s * (1.0 + zp * (1.0 - s)))
    return loss, g


def normalised_targets(E, mu, sc):
    """Y[i, b] = (E[b, i] - mu_b) / sc_b for E (nout, n)."""
    return ((np.asarray(E).T - np.asarray(mu)[None, :]) / np.asarray(sc)[None, :])


def adam_step(p, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update at step t (1-based)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def forward_bf16(params, shapes, X):
    """Normalised outputs of the tensor-core inference: BF16 inputs, weights and hidden activations,
    wide accumulation, FP32 bias and activation."""
    Ws, bs = unpack(params, shapes)
    h = bf16_round(X)
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = h @ bf16_round(W) + b
        h = bf16_round(z * _sig(z)) if l < len(Ws) - 1 else z
    return h


def predict(params, shapes, fvec, x, mu, sc):
    """Denormalised band energies (nout, n) at the points x (3, n)."""
    out, _ = forward(params, shapes, features(fvec, x))
    return (out * np.asarray(sc)[None, :] + np.asarray(mu)[None, :]).T


# ---- plain window test -----------------------------------------------------------------------
def band_energies(op_r, nw, irvec, x):
    """Ascending band energies (nw, n) of H(x) (ZHEEV on the upper triangle)."""
    hk = O.fourier_batched(op_r, nw * nw, irvec, np.asarray(x, dtype=np.float64).reshape(3, -1))
    return O.eigvals_batched(np.asfortranarray(hk.reshape(nw, nw, -1, order="F")))


def window_ranges(E, wmin, wmax):
    """(band_min, band_max) per column of E, 1-based, 0 / 0 when empty (`src/filter.jl:19`)."""
    nk = E.shape[1]
    bmin = np.zeros(nk, dtype=np.int64)
    bmax = np.zeros(nk, dtype=np.int64)
    for k in range(nk):
        s, t = O.inside_window(E[:, k], wmin, wmax)
        if t >= s:
            bmin[k], bmax[k] = s, t
    return bmin, bmax


def pair_window(op_r, nw, irvec, xk, xq, wmin, wmax):
    """Kept pairs p = ik * nq + iq (ascending) with their band ranges at x_k + x_q."""
    xk = np.asarray(xk, dtype=np.float64).reshape(3, -1)
    xq = np.asarray(xq, dtype=np.float64).reshape(3, -1)
    nk, nq = xk.shape[1], xq.shape[1]
    x = (xk[:, :, None] + xq[:, None, :]).reshape(3, nk * nq)
    E = band_energies(op_r, nw, irvec, x)
    bmin, bmax = window_ranges(E, wmin, wmax)
    keep = np.nonzero(bmin > 0)[0]
    return keep.astype(np.int64), bmin[keep], bmax[keep], E
