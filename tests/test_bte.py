"""SERTA Boltzmann consumer vs the CPU oracle (small commensurate grids).

Tolerances: per-state inverse lifetimes rtol 1e-9 (FP64 end to end; the exponentials of the
occupations amplify last-bit differences of energies by up to (e - mu) / kT), conductivity tensor
rtol 1e-9 of its largest entry.
"""
import numpy as np
import pytest

from oracle import bte_oracle as BO
from oracle import epb_oracle as O
from epb200 import synth


@pytest.mark.parametrize("ng", [3, 4])
def test_oracle_serta_symmetric_positive(ng):
    m = synth.make_model(4, 1, 1, 1, seed=5)
    x, _ = BO.grid_points(ng)
    E = O.eigvals_batched(np.asfortranarray(O.fourier_batched(m.el_ham.op_r, 16, m.el_ham.irvec, x).reshape(4, 4, -1, order="F")))
    ef = float(np.median(E[1]))
    sig, itau, info = BO.serta(m, ng, ef - 1.0, ef + 1.0, ef, 0.05, 0.05)
    assert np.allclose(sig, sig.T, rtol=1e-12, atol=0)
    assert np.all(np.linalg.eigvalsh(sig) >= -1e-12 * np.abs(sig).max())
    assert len(itau) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("nw,natom,ng,method", [(4, 1, 4, 5), (6, 2, 4, 1), (8, 1, 5, 5)])
def test_gpu_serta_vs_oracle(gpu_lib, nw, natom, ng, method):
    from epb200 import bte, pipeline

    m = synth.make_model(nw, natom, 1, 1, seed=40 + nw)
    x, _ = BO.grid_points(ng)
    E = O.eigvals_batched(np.asfortranarray(
        O.fourier_batched(m.el_ham.op_r, nw * nw, m.el_ham.irvec, x).reshape(nw, nw, -1, order="F")))
    ef = float(np.median(E[nw // 2]))
    wmin, wmax, T, eta = ef - 0.8, ef + 0.8, 0.08, 0.06
    ref, itau_ref, info = BO.serta(m, ng, wmin, wmax, ef, T, eta, method=method)
    dm = pipeline.DeviceModel(m)
    sig, st, itau = bte.serta(dm, ng, wmin, wmax, ef, T, eta, method=method, want_inv_tau=True, k_batch=3)
    assert st["kept_k"] == len(info["kept"])
    assert st["states"] == len(itau_ref)
    np.testing.assert_allclose(itau, itau_ref, rtol=1e-9, atol=1e-12 * np.abs(itau_ref).max())
    np.testing.assert_allclose(sig, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


@pytest.mark.gpu
def test_gpu_serta_mixed_vs_fp64(gpu_lib):
    """Mixed mode (g(k, Rp) on the tensor cores): conductivity within 1e-4 of the FP64 path, the
    accuracy required of sigma."""
    from epb200 import bte, pipeline

    m = synth.make_model(8, 2, 2, 1, seed=61)
    x, _ = BO.grid_points(5)
    E = O.eigvals_batched(np.asfortranarray(
        O.fourier_batched(m.el_ham.op_r, 64, m.el_ham.irvec, x).reshape(8, 8, -1, order="F")))
    ef = float(np.median(E[4]))
    dm = pipeline.DeviceModel(m, mixed=True)
    args = (dm, 5, ef - 0.8, ef + 0.8, ef, 0.08, 0.06)
    s64, st64, it64 = bte.serta(*args, prec=bte.PREC_FP64, want_inv_tau=True)
    smx, stmx, itmx = bte.serta(*args, prec=1, want_inv_tau=True)
    assert st64 == stmx
    assert np.max(np.abs(smx - s64)) <= 1e-4 * np.abs(s64).max()
    np.testing.assert_allclose(itmx, it64, rtol=1e-4, atol=1e-6 * np.abs(it64).max())


@pytest.mark.gpu
@pytest.mark.parametrize("k_batch,pair_chunk", [(2, 256), (7, 128), (32, 0)])
def test_gpu_serta_mixed_grouped(gpu_lib, k_batch, pair_chunk):
    """The grouped tensor-core kR->kq (pairs of several kept k per launch, each padded to 128 columns,
    a kept k split across column chunks when pair_chunk is small) gives the same rates as the FP64
    path within the mixed tolerance, for any batching."""
    from epb200 import bte, pipeline

    m = synth.make_model(8, 2, 2, 1, seed=62)
    ng = 8
    x, _ = BO.grid_points(ng)
    E = O.eigvals_batched(np.asfortranarray(
        O.fourier_batched(m.el_ham.op_r, 64, m.el_ham.irvec, x).reshape(8, 8, -1, order="F")))
    ef = float(np.median(E[4]))
    dm = pipeline.DeviceModel(m, mixed=True)
    args = (dm, ng, ef - 1.0, ef + 1.0, ef, 0.08, 0.06)
    s64, st64, it64 = bte.serta(*args, prec=bte.PREC_FP64, want_inv_tau=True)
    smx, stmx, itmx = bte.serta(*args, prec=1, want_inv_tau=True, k_batch=k_batch, pair_chunk=pair_chunk)
    assert st64 == stmx and stmx["pairs"] > 128 * stmx["kept_k"] // 4
    assert np.max(np.abs(smx - s64)) <= 1e-4 * np.abs(s64).max()
    np.testing.assert_allclose(itmx, it64, rtol=1e-4, atol=1e-6 * np.abs(it64).max())


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_gpu_serta_shards_add_up(gpu_lib, prec):
    """k-sharded runs (one process here, three shards): the shards' sigmas sum to the whole-grid sigma, their
    rates concatenate to the whole list, and the pair and state counts add up."""
    from epb200 import bte, pipeline

    m = synth.make_model(8, 2, 2, 1, seed=63)
    ng = 6
    x, _ = BO.grid_points(ng)
    E = O.eigvals_batched(np.asfortranarray(
        O.fourier_batched(m.el_ham.op_r, 64, m.el_ham.irvec, x).reshape(8, 8, -1, order="F")))
    ef = float(np.median(E[4]))
    dm = pipeline.DeviceModel(m, mixed=prec == 1)
    args = (dm, ng, ef - 1.0, ef + 1.0, ef, 0.08, 0.06)
    s_all, st_all, it_all = bte.serta(*args, prec=prec, want_inv_tau=True, k_batch=5)
    parts = [bte.serta(*args, prec=prec, want_inv_tau=True, k_batch=5, shard=(r, 3)) for r in range(3)]
    assert sum(p[1]["pairs"] for p in parts) == st_all["pairs"]
    assert sum(p[1]["states"] for p in parts) == st_all["states"]
    assert all(p[1]["kept_k"] == st_all["kept_k"] for p in parts)
    np.testing.assert_allclose(sum(p[0] for p in parts), s_all, rtol=1e-10, atol=1e-12 * np.abs(s_all).max())
    np.testing.assert_allclose(np.concatenate([p[2] for p in parts]), it_all, rtol=1e-10,
                               atol=1e-14 * np.abs(it_all).max())


@pytest.mark.gpu
def test_gpu_serta_more_shards_than_kept_k(gpu_lib):
    """More shards than kept k: the surplus shards have empty ranges (sigma 0, no pairs or states), the
    shards still add up to the whole, and a rank outside 0 .. count - 1 is rejected."""
    from epb200 import bte, pipeline

    m = synth.make_model(8, 2, 2, 1, seed=64)
    ng = 4
    x, _ = BO.grid_points(ng)
    E = O.eigvals_batched(np.asfortranarray(
        O.fourier_batched(m.el_ham.op_r, 64, m.el_ham.irvec, x).reshape(8, 8, -1, order="F")))
    ef = float(np.median(E[4]))
    dm = pipeline.DeviceModel(m, mixed=False)
    args = (dm, ng, ef - 0.05, ef + 0.05, ef, 0.08, 0.06)
    s_all, st_all, it_all = bte.serta(*args, prec=0, want_inv_tau=True)
    nk = st_all["kept_k"]
    assert 0 < nk < 40
    count = nk + 3
    parts = [bte.serta(*args, prec=0, want_inv_tau=True, shard=(r, count)) for r in range(count)]
    empty = [p for p in parts if p[1]["pairs"] == 0]
    assert len(empty) >= 3
    for p in empty:
        assert p[1]["states"] == 0 and not np.any(p[0])
    assert sum(p[1]["pairs"] for p in parts) == st_all["pairs"]
    np.testing.assert_allclose(sum(p[0] for p in parts), s_all, rtol=1e-10, atol=1e-12 * np.abs(s_all).max())
    np.testing.assert_allclose(np.concatenate([p[2] for p in parts]), it_all, rtol=1e-10,
                               atol=1e-14 * np.abs(it_all).max())
    with pytest.raises(Exception):
        bte.serta(*args, prec=0, shard=(count, count))
