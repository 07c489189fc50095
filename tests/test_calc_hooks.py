"""Calculator hooks of the batched loop vs the CPU oracle: eph_window_scatter! (and the uniqueness of
its target slots, the round-trip test the reference's docstring asks for) and bte_window_accumulate!
for every occupation method (bit-exact scatter; accumulation rtol 1e-12)."""
import numpy as np
import pytest

from oracle import epb_oracle as O


def _setup(rng, nbkq=5, nbk=4, nm=3, nqb=7, nkq=9, n_i=30, n_f=40):
    g2 = rng.random((nbkq, nbk, nm, nqb)) * 1e-3
    om = rng.random((nm, nqb)) * 0.01 + 1e-4
    om[0, 0] = 1e-9  # below the cutoff
    imap_i = np.array([0, 3, 7, 12][:nbk] + [0] * max(0, nbk - 4), dtype=np.int64)
    imap_f = np.zeros((nbkq, nkq), dtype=np.int64)
    fs = rng.permutation(n_f)[: nbkq * nkq] + 1
    mask = rng.random((nbkq, nkq)) < 0.7
    imap_f[mask] = fs[: mask.sum()]
    ikqs = rng.integers(1, nkq + 1, nqb).astype(np.int64)
    ikqs = rng.permutation(nkq)[:nqb] + 1  # distinct k+q per batch: unique slots
    return g2, om, imap_i, imap_f, ikqs.astype(np.int64)


def test_oracle_scatter_slots_unique():
    rng = np.random.default_rng(0)
    g2, om, imap_i, imap_f, ikqs = _setup(rng)
    n = 3 * 20 * 40
    out = np.full(n, np.nan)
    O.eph_window_scatter(out, out.copy(), g2, imap_i, imap_f, ikqs, om, 20, 0)
    # every written slot corresponds to exactly one (m, n, nu, j)
    slots = []
    for j in range(g2.shape[3]):
        for nu in range(3):
            for nn in range(g2.shape[1]):
                for m in range(g2.shape[0]):
                    i, f = imap_i[nn], imap_f[m, ikqs[j] - 1]
                    if i > 0 and f > 0:
                        slots.append(nu + 3 * (i - 1) + 3 * 20 * (f - 1))
    assert len(slots) == len(set(slots)) == np.count_nonzero(~np.isnan(out))


@pytest.mark.gpu
def test_gpu_window_scatter(gpu_lib):
    import torch

    from epb200 import batched as B

    rng = np.random.default_rng(1)
    g2, om, imap_i, imap_f, ikqs = _setup(rng)
    nm, ni_stride, i0 = 3, 16, 2
    n = nm * ni_stride * 40
    ref_g, ref_o = np.zeros(n), np.zeros(n)
    O.eph_window_scatter(ref_g, ref_o, g2, imap_i, imap_f, ikqs, om, ni_stride, i0)
    dg, do = torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64, device="cuda")
    B.eph_window_scatter(dg, do, B.jl(g2), B.jl(imap_i), B.jl(imap_f), B.jl(ikqs), B.jl(om), ni_stride, i0)
    np.testing.assert_array_equal(dg.cpu().numpy(), ref_g)
    np.testing.assert_array_equal(do.cpu().numpy(), ref_o)


@pytest.mark.gpu
@pytest.mark.parametrize("method", [1, 2, 3, 4, 5, 6])
def test_gpu_bte_window_accumulate(gpu_lib, method):
    from epb200 import batched as B

    rng = np.random.default_rng(10 + method)
    g2, om, imap_i, imap_f, ikqs = _setup(rng)
    n_i, n_f, nT, i0 = 30, 40, 2, 2
    e_i = rng.normal(0, 0.01, n_i)
    e_f = rng.normal(0, 0.01, n_f)
    wf = rng.random(n_f) / 40
    mus, ts, etas = np.array([0.0, 0.002]), np.array([0.002, 0.004]), np.array([0.003, 0.006])
    sout0 = rng.random((n_i, nT))
    ref_out, ref_in = sout0.copy(), np.zeros((14, n_f, nT))
    O.bte_window_accumulate(ref_out, ref_in, g2, om, imap_i, imap_f, ikqs, e_i, e_f, wf, mus, ts, etas, method, 1e-7, i0)
    d_out, d_in = B.jl(sout0), B.jl(np.zeros((14, n_f, nT)))
    B.bte_window_accumulate(d_out, d_in, B.jl(g2), B.jl(om), B.jl(imap_i), B.jl(imap_f), B.jl(ikqs), B.jl(e_i),
                            B.jl(e_f), B.jl(wf), B.jl(mus), B.jl(ts), B.jl(etas), method, 1e-7, i0)
    np.testing.assert_allclose(B.host(d_out), ref_out, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(B.host(d_in), ref_in, rtol=1e-12, atol=1e-300)
