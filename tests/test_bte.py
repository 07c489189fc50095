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
