"""The whole e-ph pass: CPU batched port vs the per-pair oracle (CPU), and the GPU pass vs both.

Comparisons of g2 per band are gauge-sensitive only through degenerate bands; random models have
none, so per-band values are compared directly, and band/q sums (gauge invariant) tightly.
"""
import numpy as np
import pytest

from oracle import cpu_pass, epb_oracle as O
from epb200 import synth


def _small(seed=21, nw=6, natom=2):
    return synth.config2_model(seed=seed, n_el=2, n_ph=1, nw=nw, natom=natom)


def test_cpu_pass_matches_per_pair_oracle():
    m = _small()
    xks = synth.random_kpoints(3, 1)
    xqs = synth.random_kpoints(10, 2)
    res = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=3)
    pairs = O.eph_pairs(m, xks, xqs, [(k, q) for k in range(3) for q in range(10)])
    for k in range(3):
        tot = sum(p["g2"].sum(axis=(0, 1)) for p in pairs if p["ik"] == k)
        np.testing.assert_allclose(res["g2sum"][:, k], tot, rtol=1e-10)
        for j, q in enumerate(range(0, 10, 3)):
            ref = [p for p in pairs if p["ik"] == k and p["iq"] == q][0]["g2"]
            np.testing.assert_allclose(res["g2_sample"][:, :, :, j, k], ref, rtol=1e-8, atol=1e-12 * ref.max())


@pytest.mark.gpu
@pytest.mark.parametrize("nw,natom,nk,nq,kb", [(6, 2, 7, 40, 3), (16, 4, 5, 64, 2)])
def test_gpu_pass_fp64(gpu_lib, nw, natom, nk, nq, kb):
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=31, n_el=2, n_ph=1, nw=nw, natom=natom)
    xks = synth.random_kpoints(nk, 3)
    xqs = synth.random_kpoints(nq, 4)
    dm = pipeline.DeviceModel(m)
    r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_FP64, k_batch=kb, sample_stride=7)
    ref = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=7)
    np.testing.assert_allclose(host(r.ek), ref["ek"], atol=1e-11 * np.abs(ref["ek"]).max())
    np.testing.assert_allclose(host(r.omega), ref["omega"], rtol=1e-10)
    np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-9)
    s, sr = host(r.g2_sample), ref["g2_sample"]
    np.testing.assert_allclose(s, sr, rtol=1e-7, atol=1e-10 * sr.max())
    assert r.n_elements == nk * nq * nw * nw * 3 * natom
