"""H(k+q) of the mixed pass as (H(R) rows modulated by k) x (q phases), restated in numpy (no GPU).

The pass computes H(k+q) = sum_R [H_R exp(2 pi i R.k)] exp(2 pi i R.q) on the tensor cores: the A operand
holds, per k, the Hermitian-packed rows Re H_ij (i <= j) then Im H_ij (i < j) of the modulated operator
over the K axis [cos coefficients | sin coefficients], and the B operand the q list's [cos | sin] phase
columns, packed once per pass. This checks that layout and the factorisation against the oracle's direct
Fourier sum at k + q (`src/wannier/batched_fourier_core.jl:117-139`).
"""
import numpy as np

from epb200 import synth
from oracle import epb_oracle as O


def packed_rows(nw):
    """(i, j, part) of each packed row: Re of the upper triangle column by column, then Im of the strict one."""
    rows = [(i, j, 0) for j in range(nw) for i in range(j + 1)]
    rows += [(i, j, 1) for j in range(1, nw) for i in range(j)]
    return rows


def test_hkq_from_modulated_rows_and_q_phases():
    m = synth.make_model(8, 2, 2, 1, seed=71)
    nw = 8
    op, irvec = m.el_ham.op_r, np.asarray(m.el_ham.irvec)
    rvec = irvec if irvec.shape[-1] == 3 else irvec.T  # (nr, 3)
    rng = np.random.default_rng(3)
    for _ in range(4):
        k, q = rng.random(3), rng.random(3)
        direct = O.fourier_batched(op, nw * nw, m.el_ham.irvec, (k + q)[:, None]).reshape(nw, nw, order="F")
        mod = op[: nw * nw, :] * np.exp(2j * np.pi * (rvec @ k))[None, :]   # H(R) exp(2 pi i R.k)
        ph = 2 * np.pi * (rvec @ q)
        bcol = np.concatenate([np.cos(ph), np.sin(ph)])                     # B column of q
        for (i, j, part) in packed_rows(nw):
            h = mod[i + nw * j, :]
            arow = np.concatenate([h.real, -h.imag]) if part == 0 else np.concatenate([h.imag, h.real])
            want = direct[i, j].real if part == 0 else direct[i, j].imag
            assert abs(arow @ bcol - want) <= 1e-12 * max(1.0, np.abs(direct).max())
